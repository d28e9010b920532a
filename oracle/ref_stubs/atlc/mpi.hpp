#pragma once
#include "stub_common.hpp"
namespace atlc
{
// One process on one node: node 0, local rank = rank.
inline void group_by_hostname(int proc_num, int num_procs, std::string &hostname, int &node_number,
                              int &node_local_rank, int &node_count)
{
    (void)num_procs;
    char buf[256] = {0};
    gethostname(buf, sizeof(buf) - 1);
    hostname = buf;
    node_number = 0;
    node_local_rank = proc_num;
    node_count = 1;
}
} // namespace atlc
