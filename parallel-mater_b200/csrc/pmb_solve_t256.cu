// SPDX-License-Identifier: MIT
// The group-per-body solve kernel for 256-thread CTAs: every feature set, plain
// and timed (one translation unit per CTA size, so they compile in parallel).
#include "pmb_solve_kernel.cuh"

namespace pmb {

template <bool Timed>
static void fill_builds(const void* (&out)[kSolveFeatures]) {
    out[0] = reinterpret_cast<const void*>(&k_solve<256, Timed, 0>);
    out[1] = reinterpret_cast<const void*>(&k_solve<256, Timed, 1>);
    out[2] = reinterpret_cast<const void*>(&k_solve<256, Timed, 2>);
    out[3] = reinterpret_cast<const void*>(&k_solve<256, Timed, 3>);
}

SolveVariant solve_group_variant_256() {
    SolveVariant v{};
    fill_builds<false>(v.ptr);
    fill_builds<true>(v.timed);
    v.threads = 256;
    v.smem = kWarpStage * (256 / 32);
    return v;
}

}  // namespace pmb
