// gf_field.cuh -- field accessors (HBM layouts) shared by all kernels.
//
// RefField: the reference device layout GpuPattern (access_pattern/GpuPattern.hxx:53-56):
//   U[s + V*(c + 2*(j + 3*(i + 3*mu)))], 18 reals per link, parity-split site index s.
//   Rows 0,1 of link (s,mu) are the 12 planes mu*18 + 0..11; every plane is contiguous in s, so
//   the 8 consecutive sites a warp handles per direction read 8 consecutive reals per plane.
// PackedField: this library's working layout, rows 0,1 only, in 16-byte vectors:
//   FP32: float4 planes P[(mu*3 + k)*V + s], k = 0..2 (reals 4k..4k+3 of the 12)
//   FP64: double2 planes P[(mu*6 + k)*V + s], k = 0..5 (one complex element each)
//   so a link moves with 3 (FP32) or 6 (FP64) 128-bit loads, each coalesced over the site index.
// The 12 reals of a link are ordered r[2*(3*i + j) + c] (row i, column j, c = re/im) in both.
#pragma once

#include "gf_device.cuh"

namespace gfb {

template <typename R>
struct RefField {
    R *U;
    int64_t V;
    __device__ __forceinline__ void load12(int64_t s, int mu, R r[12]) const
    {
        const R *p = U + (int64_t)mu * 18 * V + s;
#pragma unroll
        for (int k = 0; k < 12; k++) r[k] = p[k * V];
    }
    __device__ __forceinline__ void store12(int64_t s, int mu, const R r[12]) const
    {
        R *p = U + (int64_t)mu * 18 * V + s;
#pragma unroll
        for (int k = 0; k < 12; k++) p[k * V] = r[k];
    }
    // full 3x3 store (row 2 included), used by reprojection / export / random start
    __device__ __forceinline__ void store18(int64_t s, int mu, const Link<R> &L) const
    {
        R *p = U + (int64_t)mu * 18 * V + s;
#pragma unroll
        for (int i = 0; i < 3; i++)
#pragma unroll
            for (int j = 0; j < 3; j++) {
                p[(2 * (3 * i + j)) * V] = L.e[i][j].x;
                p[(2 * (3 * i + j) + 1) * V] = L.e[i][j].y;
            }
    }
};

template <typename R>
struct PackedField;

template <>
struct PackedField<float> {
    float4 *P;
    int64_t V;
    __device__ __forceinline__ void load12(int64_t s, int mu, float r[12]) const
    {
        const float4 *p = P + (int64_t)mu * 3 * V + s;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float4 v = p[k * V];
            r[4 * k] = v.x;
            r[4 * k + 1] = v.y;
            r[4 * k + 2] = v.z;
            r[4 * k + 3] = v.w;
        }
    }
    __device__ __forceinline__ void store12(int64_t s, int mu, const float r[12]) const
    {
        float4 *p = P + (int64_t)mu * 3 * V + s;
#pragma unroll
        for (int k = 0; k < 3; k++) p[k * V] = make_float4(r[4 * k], r[4 * k + 1], r[4 * k + 2], r[4 * k + 3]);
    }
};

template <>
struct PackedField<double> {
    double2 *P;
    int64_t V;
    __device__ __forceinline__ void load12(int64_t s, int mu, double r[12]) const
    {
        const double2 *p = P + (int64_t)mu * 6 * V + s;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const double2 v = p[k * V];
            r[2 * k] = v.x;
            r[2 * k + 1] = v.y;
        }
    }
    __device__ __forceinline__ void store12(int64_t s, int mu, const double r[12]) const
    {
        double2 *p = P + (int64_t)mu * 6 * V + s;
#pragma unroll
        for (int k = 0; k < 6; k++) p[k * V] = make_double2(r[2 * k], r[2 * k + 1]);
    }
};

// The packed layout read through L2 only (ld.global.cg).  A kernel that updates the field in one
// pass and reads it in the next -- the persistent chunk kernel -- uses it: another SM may have
// rewritten a line this SM still holds in its (non-coherent) L1 since the previous pass.
template <typename R>
struct PackedFieldL2;

template <>
struct PackedFieldL2<float> {
    float4 *P;
    int64_t V;
    __device__ __forceinline__ void load12(int64_t s, int mu, float r[12]) const
    {
        const float4 *p = P + (int64_t)mu * 3 * V + s;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const float4 v = __ldcg(p + k * V);
            r[4 * k] = v.x;
            r[4 * k + 1] = v.y;
            r[4 * k + 2] = v.z;
            r[4 * k + 3] = v.w;
        }
    }
    __device__ __forceinline__ void store12(int64_t s, int mu, const float r[12]) const
    {
        PackedField<float>{P, V}.store12(s, mu, r);
    }
};

template <>
struct PackedFieldL2<double> {
    double2 *P;
    int64_t V;
    __device__ __forceinline__ void load12(int64_t s, int mu, double r[12]) const
    {
        const double2 *p = P + (int64_t)mu * 6 * V + s;
#pragma unroll
        for (int k = 0; k < 6; k++) {
            const double2 v = __ldcg(p + k * V);
            r[2 * k] = v.x;
            r[2 * k + 1] = v.y;
        }
    }
    __device__ __forceinline__ void store12(int64_t s, int mu, const double r[12]) const
    {
        PackedField<double>{P, V}.store12(s, mu, r);
    }
};

template <typename R, class F>
__device__ __forceinline__ void load_link(const F &f, int64_t s, int mu, Link<R> &L)
{
    R r[12];
    f.load12(s, mu, r);
    unpack12(L, r);
    reconstruct(L);
}

template <typename R, class F>
__device__ __forceinline__ void store_link(const F &f, int64_t s, int mu, const Link<R> &L)
{
    R r[12];
    pack12(L, r);
    f.store12(s, mu, r);
}

// the Philox key the reference gives the (mu = 0, up) thread of site h of a parity half:
// blockIdx.x*blockDim.x + threadIdx.x with 32 sites and 256 threads per block (apps/Makefile:36,
// LandauKernelsSU3.hxx:225-230,272)
__device__ __forceinline__ uint32_t ref_rng_tid(int64_t h) { return (uint32_t)((h >> 5) * 256 + (h & 31)); }

}  // namespace gfb
