// Exposes the reference's MortonCode3D / MortonCode6D (Framework/morton.h, included unchanged
// from the reference tree) through plain C symbols so the tests can pin the oracle's and the
// GPU's Morton codes against the reference's own code.  Test infrastructure only.
#include <cuda_runtime.h>

#include <iostream>

#include "morton.h"

extern "C" void ref_morton3d(const float* xyz, int n, uint32_t* out) {
    MortonCode3D m;
    for (int i = 0; i < n; ++i) out[i] = m(make_float3(xyz[3 * i], xyz[3 * i + 1], xyz[3 * i + 2]));
}

// MortonCode6D returns 64 bits; the reference stores it into a uint32_t vector (MC_SIZE,
// bvh.h:17), which keeps the low 32 bits.
extern "C" void ref_morton6d_u32(const float* a, const float* b, int n, uint32_t* out) {
    MortonCode6D m;
    for (int i = 0; i < n; ++i)
        out[i] = (uint32_t)m(make_float3(a[3 * i], a[3 * i + 1], a[3 * i + 2]),
                             make_float3(b[3 * i], b[3 * i + 1], b[3 * i + 2]));
}
