// The marker section of the reference's binary output file, written from and
// read into the device-resident markers.
//
// saver() (loadmart.c:795-808) writes per marker nine 4-byte floats (x, y, T,
// eta, hi, por, grain size, tmax, accretion time) and three bytes (magnetisation
// state, magnetisation time converted to char, type): 39 bytes, no padding, in
// the caller's marker order.  loader() (loadmart.c:521-535) reads the floats
// back and stores the last of them (the accretion time) in both magnetisation
// fields; the two magnetisation bytes of the file are dropped.
//
// 256 records are 9984 = 624 x 16 bytes, so a block of 256 caller indices owns
// a 16-byte aligned stretch of the section (when the section starts on 16
// bytes): each block assembles or takes apart its records in shared memory and
// moves the stretch with 16-byte accesses.  Markers are read from or written to
// their device slots through pos[] (caller index -> slot).
#pragma once

#include "i2g_dev.cuh"

namespace i2g {

constexpr int kPrnRecord = 39;
constexpr int kPrnBlock = 256;

// C's float-to-char conversion as x86-64 builds emit it: the low byte of the
// 32-bit truncation, whose result is INT_MIN for NaN and values outside the int
// range
__device__ __forceinline__ int8_t prn_char(double v)
{
    const int32_t i = (v > -2147483649.0 && v < 2147483648.0) ? (int32_t)v : INT32_MIN;
    return (int8_t)(uint8_t)(i & 0xff);
}

__device__ __forceinline__ void prn_put_f32(uint8_t *r, float f)
{
    const uint32_t u = __float_as_uint(f);
    r[0] = (uint8_t)u;
    r[1] = (uint8_t)(u >> 8);
    r[2] = (uint8_t)(u >> 16);
    r[3] = (uint8_t)(u >> 24);
}

__device__ __forceinline__ float prn_get_f32(const uint8_t *r)
{
    return __uint_as_float((uint32_t)r[0] | ((uint32_t)r[1] << 8) | ((uint32_t)r[2] << 16) | ((uint32_t)r[3] << 24));
}

// pos[id[i]] = i
__global__ void k_prn_pos(int64_t n, const int32_t *__restrict__ id, int32_t *__restrict__ pos)
{
    const int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) pos[id[i]] = (int32_t)i;
}

// the shared-memory stretch of a block <-> the section (16-byte moves when the
// stretch is whole and aligned)
__device__ __forceinline__ void prn_move(uint8_t *dst, const uint8_t *src, int64_t nb)
{
    const bool wide = nb == (int64_t)kPrnBlock * kPrnRecord && (((uintptr_t)dst | (uintptr_t)src) & 15) == 0;
    if (wide) {
        const uint4 *s = reinterpret_cast<const uint4 *>(src);
        uint4 *d = reinterpret_cast<uint4 *>(dst);
        for (int k = threadIdx.x; k < kPrnBlock * kPrnRecord / 16; k += blockDim.x) d[k] = s[k];
    } else {
        for (int64_t k = threadIdx.x; k < nb; k += blockDim.x) dst[k] = src[k];
    }
}

// saver()'s records of the caller's markers [0, n); fields the context does not
// keep (gr, acc: caller order, NULL = 0; mg_old, mg_time: caller order, NULL =
// the context's own when it produces them, else 0; tmax, hi, por when untracked)
// are written as 0
__global__ void __launch_bounds__(kPrnBlock) k_prn_pack(int64_t n, const int32_t *__restrict__ pos,
                                                        const __grid_constant__ MarkerView M,
                                                        const float *__restrict__ gr, const float *__restrict__ acc,
                                                        const int8_t *__restrict__ mgo,
                                                        const double *__restrict__ mgt, uint8_t *__restrict__ out)
{
    __shared__ __align__(16) uint8_t buf[kPrnBlock * kPrnRecord];
    const int64_t j0 = (int64_t)blockIdx.x * kPrnBlock;
    const int64_t j = j0 + threadIdx.x;
    if (j < n) {
        const int64_t s = pos[j];
        uint8_t *r = buf + threadIdx.x * kPrnRecord;
        prn_put_f32(r + 0, (float)M.x[s]);
        prn_put_f32(r + 4, (float)M.y[s]);
        prn_put_f32(r + 8, (float)M.T[s]);
        prn_put_f32(r + 12, (float)M.eta[s]);
        prn_put_f32(r + 16, M.hi ? (float)M.hi[s] : 0.0f);
        prn_put_f32(r + 20, M.por ? (float)M.por[s] : 0.0f);
        prn_put_f32(r + 24, gr ? gr[j] : 0.0f);
        prn_put_f32(r + 28, M.tmax ? (float)M.tmax[s] : 0.0f);
        prn_put_f32(r + 32, acc ? acc[j] : 0.0f);
        // magnetisation: the host's arrays, else the context's own (when produced), else 0
        r[36] = (uint8_t)(mgo ? mgo[j] : (M.mgo ? M.mgo[s] : 0));
        r[37] = (uint8_t)(mgt ? prn_char(mgt[j]) : (M.mgt ? prn_char(M.mgt[s]) : 0));
        r[38] = (uint8_t)M.type[s];
    }
    __syncthreads();
    const int64_t nrec = n - j0 < kPrnBlock ? n - j0 : kPrnBlock;
    prn_move(out + j0 * kPrnRecord, buf, nrec * kPrnRecord);
}

// loader()'s arrays from the records of markers [0, n), in caller order: the
// nine floats (f[k] + j, k = x, y, T, eta, hi, por, gr, tmax, acc, stride ld),
// the type byte, and the magnetisation fields as loader() leaves them
__global__ void __launch_bounds__(kPrnBlock) k_prn_unpack(int64_t n, const uint8_t *__restrict__ in,
                                                          float *__restrict__ f, int64_t ld,
                                                          int8_t *__restrict__ type, int8_t *__restrict__ mgo,
                                                          double *__restrict__ mgt)
{
    __shared__ __align__(16) uint8_t buf[kPrnBlock * kPrnRecord];
    const int64_t j0 = (int64_t)blockIdx.x * kPrnBlock;
    const int64_t nrec = n - j0 < kPrnBlock ? n - j0 : kPrnBlock;
    prn_move(buf, in + j0 * kPrnRecord, nrec * kPrnRecord);
    __syncthreads();
    const int64_t j = j0 + threadIdx.x;
    if (j >= n) return;
    const uint8_t *r = buf + threadIdx.x * kPrnRecord;
#pragma unroll
    for (int k = 0; k < 9; k++) f[k * ld + j] = prn_get_f32(r + 4 * k);
    const float a = prn_get_f32(r + 32);
    type[j] = (int8_t)r[38];
    mgo[j] = prn_char((double)a);
    mgt[j] = (double)a;
}

// caller-order FP32 field -> device-order FP64 field (dst[s] = src[id[s]])
__global__ void k_prn_sortin(int64_t n, const int32_t *__restrict__ id, const float *__restrict__ src,
                             double *__restrict__ dst)
{
    const int64_t s = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (s < n) dst[s] = (double)src[id[s]];
}

}  // namespace i2g
