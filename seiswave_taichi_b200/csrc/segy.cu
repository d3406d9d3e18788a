// segy.cu -- SEG-Y trace decoding on the device: the samples of every trace,
// big-endian as the standard stores them, to float32, plus each trace's
// SourceX header word.  The reference reads models and shot records with
// segyio (ReadSegy.py:3-18), which is not part of this build; the file's
// bytes are copied to the device once and decoded here.
//
// Layout after the 3600-byte file header (and any extended textual headers,
// which the caller skips): ntraces records of a 240-byte trace header
// followed by nsamples samples.  Sample formats (binary header bytes
// 3225-3226): 1 IBM hexadecimal float, 2 int32, 3 int16, 5 IEEE float,
// 8 int8.  SourceX is the big-endian int32 at trace-header bytes 73-76.
//
// IBM float: sign bit, 7-bit excess-64 base-16 exponent e and 24-bit
// fraction f, value (-1)^s * f * 2^(4(e-64)-24).  f < 2^24 and the exponent
// fits a double, so the value is exact in double and rounds once to float
// (subnormal results and the overflow to infinity included); a zero fraction
// gives a zero of that sign.  The work is byte traffic: one thread per sample,
// consecutive threads on consecutive samples of a trace.
#include <cstdint>
#include <cuda_runtime.h>

namespace sw {

// When the value is a normal float its 24-bit fraction, shifted left until
// bit 23 is set, is the float significand as it is: the bits are assembled
// directly.  Values that would be subnormal or overflow take the double route.
__device__ __forceinline__ float ibm_to_float(uint32_t w) {
  const uint32_t f = w & 0x00ffffffu;
  const uint32_t sign = w & 0x80000000u;
  if (f == 0) return __uint_as_float(sign);
  const int e = (int)((w >> 24) & 0x7fu);
  const int lz = __clz(f) - 8;            // f << lz lies in [2^23, 2^24)
  const int ex = 4 * (e - 64) - 1 - lz;   // value = 1.m * 2^ex
  if (ex >= -126 && ex <= 127)
    return __uint_as_float(sign | ((uint32_t)(ex + 127) << 23) | ((f << lz) & 0x007fffffu));
  const double v = ldexp((double)f, 4 * (e - 64) - 24);
  return __double2float_rn(sign ? -v : v);
}

template <int BPS>
__device__ __forceinline__ uint32_t raw_word(const unsigned char* p) {
  if (BPS == 4) return *reinterpret_cast<const uint32_t*>(p);
  if (BPS == 2) return ((uint32_t)p[0] << 8) | p[1];
  return p[0];
}

template <int FMT>
__device__ __forceinline__ float decode_raw(uint32_t r) {
  if (FMT == 1) return ibm_to_float(__byte_perm(r, 0, 0x0123));
  if (FMT == 5) return __uint_as_float(__byte_perm(r, 0, 0x0123));
  if (FMT == 2) return (float)(int32_t)__byte_perm(r, 0, 0x0123);
  if (FMT == 3) return (float)(int16_t)(uint16_t)r;
  return (float)(int8_t)(uint8_t)r;
}

// grid: x over the samples of a trace, y over traces (both grid-stride).
// Each thread loads four samples one grid stride apart before decoding them,
// so every load stays coalesced and four are in flight per thread.
template <int FMT>
__global__ void k_segy_decode(const unsigned char* __restrict__ src, long long ntraces, int nsamples,
                              float* __restrict__ out, int32_t* __restrict__ srcx) {
  constexpr int BPS = (FMT == 3) ? 2 : (FMT == 8) ? 1 : 4;
  constexpr int U = 4;
  const long long rec = 240 + (long long)BPS * nsamples;
  const int stride = gridDim.x * blockDim.x;
  for (long long t = blockIdx.y; t < ntraces; t += gridDim.y) {
    const unsigned char* tr = src + t * rec;
    float* o = out + t * nsamples;
    // 32-bit samples whose trace and output row are 16-byte aligned (every
    // trace when nsamples is a multiple of 4): four samples per 16-byte load
    // and store, two such vectors in flight per thread; the scalar loop below
    // takes the rest of the row and every other case
    int done = 0;
    if (BPS == 4 && ((reinterpret_cast<uintptr_t>(tr + 240) | reinterpret_cast<uintptr_t>(o)) & 15) == 0) {
      const int nv = nsamples >> 2;
      const uint4* in4 = reinterpret_cast<const uint4*>(tr + 240);
      float4* out4 = reinterpret_cast<float4*>(o);
      for (int v0 = blockIdx.x * blockDim.x + threadIdx.x; v0 < nv; v0 += 2 * stride) {
        uint4 w[2];
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int v = v0 + u * stride;
          w[u] = v < nv ? in4[v] : make_uint4(0, 0, 0, 0);
        }
#pragma unroll
        for (int u = 0; u < 2; ++u) {
          const int v = v0 + u * stride;
          if (v < nv)
            out4[v] = make_float4(decode_raw<FMT>(w[u].x), decode_raw<FMT>(w[u].y), decode_raw<FMT>(w[u].z),
                                  decode_raw<FMT>(w[u].w));
        }
      }
      done = nv << 2;
    }
    for (int s0 = done + blockIdx.x * blockDim.x + threadIdx.x; s0 < nsamples; s0 += U * stride) {
      uint32_t r[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int s = s0 + u * stride;
        r[u] = s < nsamples ? raw_word<BPS>(tr + 240 + (long long)BPS * s) : 0u;
      }
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int s = s0 + u * stride;
        if (s < nsamples) o[s] = decode_raw<FMT>(r[u]);
      }
    }
    // byte by byte: with 16- or 8-bit samples a record need not keep 4-byte alignment
    if (srcx && blockIdx.x == 0 && threadIdx.x == 0)
      srcx[t] = (int32_t)(((uint32_t)tr[72] << 24) | ((uint32_t)tr[73] << 16) | ((uint32_t)tr[74] << 8) | tr[75]);
  }
}

cudaError_t segy_decode(const void* src, long long ntraces, int nsamples, int format, float* out, int32_t* srcx,
                        cudaStream_t st) {
  if (ntraces == 0 || nsamples == 0) return cudaSuccess;
  // 256-thread blocks, one per 1024 samples of a trace (16 per trace at
  // 16000 samples): one 16-byte vector per thread on aligned traces
  const int gx = (int)((nsamples + 1023) / 1024 < 64 ? (nsamples + 1023) / 1024 : 64);
  const dim3 grid(gx, (unsigned)(ntraces < 65535 ? ntraces : 65535));
  const unsigned char* b = static_cast<const unsigned char*>(src);
  switch (format) {
    case 1: k_segy_decode<1><<<grid, 256, 0, st>>>(b, ntraces, nsamples, out, srcx); break;
    case 2: k_segy_decode<2><<<grid, 256, 0, st>>>(b, ntraces, nsamples, out, srcx); break;
    case 3: k_segy_decode<3><<<grid, 256, 0, st>>>(b, ntraces, nsamples, out, srcx); break;
    case 5: k_segy_decode<5><<<grid, 256, 0, st>>>(b, ntraces, nsamples, out, srcx); break;
    case 8: k_segy_decode<8><<<grid, 256, 0, st>>>(b, ntraces, nsamples, out, srcx); break;
    default: return cudaErrorInvalidValue;
  }
  return cudaGetLastError();
}

}  // namespace sw
