// Shared helpers for the gm_b200 CUDA sources (sm_100a).
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/gm_b200.h"

namespace gm {

// Records the last CUDA error string for gm_last_error().
void set_error(const char *where, cudaError_t err);
void set_error_msg(const char *msg);

inline int check_launch(const char *where)
{
    cudaError_t err = cudaGetLastError();
    if (err != cudaSuccess) {
        set_error(where, err);
        return GM_ERR_LAUNCH;
    }
    return GM_OK;
}

inline cudaStream_t as_stream(void *s) { return reinterpret_cast<cudaStream_t>(s); }

template <typename T> struct vec2;
template <> struct vec2<double> { using type = double2; };
template <> struct vec2<float> { using type = float2; };

template <typename T2>
__device__ __forceinline__ T2 cmul(T2 a, T2 b)
{
    T2 r;
    r.x = a.x * b.x - a.y * b.y;
    r.y = a.x * b.y + a.y * b.x;
    return r;
}

template <typename T2>
__device__ __forceinline__ T2 cadd(T2 a, T2 b)
{
    T2 r;
    r.x = a.x + b.x;
    r.y = a.y + b.y;
    return r;
}

template <typename T2>
__device__ __forceinline__ T2 csub(T2 a, T2 b)
{
    T2 r;
    r.x = a.x - b.x;
    r.y = a.y - b.y;
    return r;
}

template <typename T2>
__device__ __forceinline__ T2 cconj(T2 a)
{
    a.y = -a.y;
    return a;
}

template <typename T2, typename T>
__device__ __forceinline__ T2 make2(T x, T y)
{
    T2 r;
    r.x = x;
    r.y = y;
    return r;
}

// Lane geometry: lane j (0-based) is north ring j (ring number j + 1); the last lane
// (j = 2 nside - 1) is the equator ring, which has no southern partner.
__host__ __device__ __forceinline__ int64_t north_ring(int64_t j) { return j; }
__host__ __device__ __forceinline__ int64_t south_ring(int64_t nside, int64_t j)
{
    return 4 * nside - 2 - j;
}
__host__ __device__ __forceinline__ int64_t ring_nphi(int64_t nside, int64_t r)
{
    int64_t ring = r + 1;
    int64_t north = ring > 2 * nside ? 4 * nside - ring : ring;
    return north < nside ? 4 * north : 4 * nside;
}
__host__ __device__ __forceinline__ int64_t ring_offset(int64_t nside, int64_t r)
{
    // first pixel of ring r (RING scheme), matching cumsum(nphi)
    int64_t ring = r + 1;
    int64_t npix = 12 * nside * nside;
    if (ring < nside) return 2 * ring * (ring - 1);
    if (ring <= 3 * nside) return 2 * nside * (nside - 1) + (ring - nside) * 4 * nside;
    int64_t k = 4 * nside - ring;  // south cap, k in [1, nside)
    return npix - 2 * k * (k + 1);
}
// Twiddle-table segment of a ring of length nphi = 4 i: entries exp(-2 pi i k / nphi), k < nphi/2.
__host__ __device__ __forceinline__ int64_t twiddle_offset(int64_t nphi)
{
    int64_t i = nphi / 4;
    return i * (i - 1);
}

}  // namespace gm
