# SPDX-License-Identifier: MIT
"""Host-side Python mirror of the B200 AVBD rigid step.

``scenes`` builds the synthetic workloads (box pyramid, box piles, capsule
chains, scene batches) as plain record arrays; ``core`` binds the CUDA
library ``libpmb200_core.so`` through its C ABI.
"""
