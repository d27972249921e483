// Target-leaf lists built on the GPU from the device pair lists of a Plan.
#pragma once

#include "devbuf.hpp"
#include "plan.hpp"

namespace ifgf
{

// The target-leaf CSR tables of Plan::build_target_lists (same entries, same
// order) for the source boxes `rank` owns (all when rank < 0), built on the
// current device: far_off / near_off hold one offset per target leaf of
// P.tleaf_gid plus the total, far_src / near_src the source global box ids.
// Uploads the pair lists first where a host walk made them.
void build_target_lists_gpu(Plan& P, int rank, DevBuf<long long>& far_off, DevBuf<int>& far_src,
                            DevBuf<long long>& near_off, DevBuf<int>& near_src);

} // namespace ifgf
