// SPDX-License-Identifier: MIT
// The group-per-body solve kernel for 384-thread CTAs: every feature set, plain
// and timed (one translation unit per CTA size, so they compile in parallel).
#include "pmb_solve_kernel.cuh"

namespace pmb {

template <bool Timed>
static void fill_builds(const void* (&out)[kSolveFeatures]) {
    out[0] = reinterpret_cast<const void*>(&k_solve<384, Timed, 0>);
    out[1] = reinterpret_cast<const void*>(&k_solve<384, Timed, 1>);
    out[2] = reinterpret_cast<const void*>(&k_solve<384, Timed, 2>);
    out[3] = reinterpret_cast<const void*>(&k_solve<384, Timed, 3>);
}

SolveVariant solve_group_variant_384() {
    SolveVariant v{};
    fill_builds<false>(v.ptr);
    fill_builds<true>(v.timed);
    v.threads = 384;
    v.smem = kWarpStage * (384 / 32);
    return v;
}

}  // namespace pmb
