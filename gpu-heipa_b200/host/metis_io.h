// METIS graph reader and partition/mapping writer.
//
// Reader contract follows src/datastructures/host_graph.h:154-247 (header
// "n m [fmt]", m undirected, 1-based neighbour ids, optional vertex weight
// first on each line, optional edge weight after each neighbour, '%' comment
// lines) with two deliberate differences: the fmt field is read as a standard
// right-aligned METIS code (a 3-digit code such as 011 means the same in both),
// and malformed input returns an error instead of exiting.
//
// Writer contract follows src/utility/util.h:288-329: one decimal block id per
// line, n lines, no header.
#pragma once
#include "hp_types.h"

namespace hp {

// Returns 0 on success; on failure returns non-zero and sets `err`.
int read_metis(const std::string &path, HostCSR &g, std::string &err);
int write_metis(const std::string &path, const HostCSR &g, bool write_vw, bool write_ew, std::string &err);
int write_partition(const std::string &path, const u32 *part, u32 n, std::string &err);
int read_partition(const std::string &path, std::vector<u32> &part, std::string &err);

} // namespace hp
