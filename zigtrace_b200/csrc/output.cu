/*
 * output.cu -- the output stage on the device: Image.toRgb8 / Output.encode
 * (src/image.zig:14-73) and png.writePng (src/png.zig:10-117).
 *
 * Both are byte work bound by memory traffic.  The encode maps each f64
 * channel to a byte in one pass.  The PNG is assembled in four launches:
 *   k_png_body    every byte of the file that does not depend on a checksum
 *                 (signature, IHDR, zlib header, stored-block headers, the
 *                 filter byte of each row, the RGB rows, IEND), one output
 *                 byte per thread, gathered from the RGB8 image;
 *   k_adler       Adler-32 of the uncompressed stream as two modular sums
 *                 (A = 1 + sum d_i, B = n + sum (n - i) d_i, mod 65521);
 *   k_crc_blocks  CRC-32 of 32 KB slices of the IDAT chunk, staged through
 *                 shared memory; slices and the bytes inside a slice are
 *                 combined with crc(A||B) = crc(A) * x^(8|B|) + crc(B)
 *                 over GF(2) modulo the CRC polynomial;
 *   k_crc_final   combines the slices and writes the chunk CRC.
 * The bytes are exactly those of the reference's writer for the same RGB8
 * input (same block split, same headers, same checksums).
 */
#include <cuda_runtime.h>
#include <math.h>
#include <string.h>

#include <string>
#include <vector>

#include "output.cuh"
#include "scene_host.h"

namespace zt {

static zt_status out_cuda_fail(cudaError_t e, const char* what) {
  return fail(ZT_ERR_CUDA, std::string(what) + ": " + cudaGetErrorString(e));
}

/* ------------------------------------------------------------- encode ---- */
/* Output.encode, image.zig:31-37, with Tonemap.apply, image.zig:14-21: the
 * same f64 operations as the host zt_image_to_rgb8. */
__device__ __forceinline__ uint8_t encode_value(double linear, uint32_t tonemap, double gamma, double exposure) {
  const double v = isnan(linear) ? 0.0 : linear;
  const double x = fmax(v * exposure, 0.0);
  double m;
  if (tonemap == 0) m = x;
  else if (tonemap == 1) m = x / (1.0 + x);
  else m = (x * (2.51 * x + 0.03)) / (x * (2.43 * x + 0.59) + 0.14);
  /* std.math.clamp: a NaN gives 1, as @min(NaN, 1) = 1.  Spelled out: nvcc
   * may turn fmax(0, fmin(x, 1)) into a saturating operation that maps NaN
   * to 0 (inf / (1 + inf) in the Reinhard curve, for one). */
  const double mapped = isnan(m) ? 1.0 : fmax(0.0, fmin(m, 1.0));
  const double corrected = pow(mapped, 1.0 / gamma);
  const double c = isnan(corrected) ? 1.0 : fmax(0.0, fmin(corrected, 1.0));
  return (uint8_t)round(c * 255.0);
}

/* Four channel values per thread: two 16-byte loads, one 4-byte store. */
__global__ void k_encode_rgb8(const double* __restrict__ px, uint64_t n, uint32_t tonemap, double gamma,
                              double exposure, uint8_t* __restrict__ out) {
  const uint64_t quads = n / 4;
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t q = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; q < quads; q += stride) {
    const double2 a = __ldcs(reinterpret_cast<const double2*>(px) + 2 * q);
    const double2 b = __ldcs(reinterpret_cast<const double2*>(px) + 2 * q + 1);
    uchar4 r;
    r.x = encode_value(a.x, tonemap, gamma, exposure);
    r.y = encode_value(a.y, tonemap, gamma, exposure);
    r.z = encode_value(b.x, tonemap, gamma, exposure);
    r.w = encode_value(b.y, tonemap, gamma, exposure);
    reinterpret_cast<uchar4*>(out)[q] = r;
  }
  const uint64_t t = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
  if (t < n - 4 * quads) out[4 * quads + t] = encode_value(px[4 * quads + t], tonemap, gamma, exposure);
}

/* The same one value per thread, for buffers without 16/4-byte alignment. */
__global__ void k_encode_rgb8_scalar(const double* __restrict__ px, uint64_t n, uint32_t tonemap, double gamma,
                                     double exposure, uint8_t* __restrict__ out) {
  const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
  for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride)
    out[i] = encode_value(px[i], tonemap, gamma, exposure);
}

static int device_sms() {
  int dev = 0, sms = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) !=
                                                cudaSuccess || sms <= 0)
    sms = 148;
  return sms;
}

/* Grid-stride launches: at most 8 blocks of 256 per SM. */
static unsigned stride_grid(uint64_t items, int block) {
  const uint64_t need = (items + block - 1) / block;
  const uint64_t cap = (uint64_t)device_sms() * 8;
  return (unsigned)(need < 1 ? 1 : (need < cap ? need : cap));
}

zt_status launch_encode_rgb8(const double* d_px, uint64_t n_values, uint32_t tonemap, double gamma, double exposure,
                             uint8_t* d_out, cudaStream_t stream) {
  if (n_values == 0) return ZT_OK;
  const bool aligned = ((uintptr_t)d_px % 16 == 0) && ((uintptr_t)d_out % 4 == 0);
  if (aligned) {
    const uint64_t quads = n_values / 4;
    k_encode_rgb8<<<stride_grid(quads > 4 ? quads : 4, 256), 256, 0, stream>>>(d_px, n_values, tonemap, gamma,
                                                                               exposure, d_out);
  } else {
    k_encode_rgb8_scalar<<<stride_grid(n_values, 256), 256, 0, stream>>>(d_px, n_values, tonemap, gamma, exposure,
                                                                          d_out);
  }
  const cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? ZT_OK : out_cuda_fail(e, "launch k_encode_rgb8");
}

/* ---------------------------------------------------------------- CRC ---- */
/* CRC-32 of PNG (ISO-HDLC: reflected polynomial 0xEDB88320, register
 * preset to all ones, result complemented).  Polynomials over GF(2) are
 * held bit-reflected: bit 31 is the coefficient of x^0. */
constexpr uint32_t kCrcPoly = 0xEDB88320u;

/* a * b mod P. */
__host__ __device__ inline uint32_t crc_mulmod(uint32_t a, uint32_t b) {
  uint32_t p = 0;
  for (uint32_t m = 1u << 31; m != 0; m >>= 1) {
    if (a & m) p ^= b;
    b = (b & 1u) ? (b >> 1) ^ kCrcPoly : b >> 1; /* b *= x */
  }
  return p;
}

struct CrcTables {
  uint32_t byte[256]; /* register update for one input byte */
  uint32_t xpow[32];  /* x^(8 * 2^k) mod P */
};

static CrcTables make_crc_tables() {
  CrcTables T;
  for (uint32_t i = 0; i < 256; ++i) {
    uint32_t c = i;
    for (int k = 0; k < 8; ++k) c = (c & 1u) ? (c >> 1) ^ kCrcPoly : c >> 1;
    T.byte[i] = c;
  }
  uint32_t x8 = 1u << 31; /* x^0 */
  for (int k = 0; k < 8; ++k) x8 = (x8 & 1u) ? (x8 >> 1) ^ kCrcPoly : x8 >> 1;
  T.xpow[0] = x8;
  for (int k = 1; k < 32; ++k) T.xpow[k] = crc_mulmod(T.xpow[k - 1], T.xpow[k - 1]);
  return T;
}

/* c * x^(8n) mod P: the register after n more zero bytes. */
__host__ __device__ inline uint32_t crc_shift(uint32_t c, uint32_t n, const uint32_t* xpow) {
  for (int k = 0; n != 0; ++k, n >>= 1)
    if (n & 1u) c = crc_mulmod(c, xpow[k]);
  return c;
}

constexpr int kCrcThreads = 256;
constexpr int kCrcSeg = 128;                      /* bytes per thread */
constexpr int kCrcSlice = kCrcThreads * kCrcSeg;  /* 32 KB per block */
constexpr int kCrcPitch = kCrcSeg + 4;            /* shared-memory pitch: consecutive threads, consecutive banks */

/* Tree-combines part[0..kCrcThreads) (with byte lengths len[]) into part[0]. */
__device__ void crc_tree(uint32_t* part, uint32_t* len, const uint32_t* xpow) {
  const int t = threadIdx.x;
  for (int s = 1; s < kCrcThreads; s <<= 1) {
    if ((t % (2 * s)) == 0 && t + s < kCrcThreads) {
      part[t] = crc_shift(part[t], len[t + s], xpow) ^ part[t + s];
      len[t] += len[t + s];
    }
    __syncthreads();
  }
}

/* Zero-preset CRC register of each 32 KB slice of data[0, n). */
__global__ void __launch_bounds__(kCrcThreads) k_crc_blocks(const uint8_t* __restrict__ data, uint32_t n,
                                                            CrcTables T, uint32_t* __restrict__ slice_crc) {
  __shared__ uint32_t tab[256];
  __shared__ uint32_t xpow[32];
  __shared__ uint8_t buf[kCrcThreads * kCrcPitch];
  __shared__ uint32_t part[kCrcThreads], len[kCrcThreads];
  const int t = threadIdx.x;
  for (int i = t; i < 256; i += kCrcThreads) tab[i] = T.byte[i];
  if (t < 32) xpow[t] = T.xpow[t];
  const uint32_t base = blockIdx.x * (uint32_t)kCrcSlice;
  const uint32_t m = n - base < (uint32_t)kCrcSlice ? n - base : (uint32_t)kCrcSlice;
  for (uint32_t i = t; i < m; i += kCrcThreads) buf[(i / kCrcSeg) * kCrcPitch + (i % kCrcSeg)] = data[base + i];
  __syncthreads();
  const uint32_t s0 = (uint32_t)t * kCrcSeg;
  const uint32_t sl = s0 < m ? (m - s0 < (uint32_t)kCrcSeg ? m - s0 : (uint32_t)kCrcSeg) : 0;
  uint32_t c = 0;
  for (uint32_t k = 0; k < sl; ++k) c = tab[(c ^ buf[t * kCrcPitch + k]) & 0xffu] ^ (c >> 8);
  part[t] = c;
  len[t] = sl;
  __syncthreads();
  crc_tree(part, len, xpow);
  if (t == 0) slice_crc[blockIdx.x] = part[0];
}

/* Combines the slice registers, presets and complements as PNG's CRC does,
 * and writes the result big-endian at out. */
__global__ void __launch_bounds__(kCrcThreads) k_crc_final(const uint32_t* __restrict__ slice_crc, uint32_t n_slices,
                                                           uint32_t n, CrcTables T, uint8_t* __restrict__ out) {
  __shared__ uint32_t xpow[32];
  __shared__ uint32_t part[kCrcThreads], len[kCrcThreads];
  const int t = threadIdx.x;
  if (t < 32) xpow[t] = T.xpow[t];
  __syncthreads();
  const uint32_t per = (n_slices + kCrcThreads - 1) / kCrcThreads;
  uint32_t c = 0, l = 0;
  for (uint32_t s = (uint32_t)t * per; s < n_slices && s < (uint32_t)(t + 1) * per; ++s) {
    const uint32_t sl = n - s * (uint32_t)kCrcSlice < (uint32_t)kCrcSlice ? n - s * (uint32_t)kCrcSlice
                                                                           : (uint32_t)kCrcSlice;
    c = crc_shift(c, sl, xpow) ^ slice_crc[s];
    l += sl;
  }
  part[t] = c;
  len[t] = l;
  __syncthreads();
  crc_tree(part, len, xpow);
  if (t == 0) {
    const uint32_t crc = ~(part[0] ^ crc_shift(0xFFFFFFFFu, n, xpow));
    out[0] = (uint8_t)(crc >> 24);
    out[1] = (uint8_t)(crc >> 16);
    out[2] = (uint8_t)(crc >> 8);
    out[3] = (uint8_t)crc;
  }
}

static uint32_t crc32_host(const uint8_t* p, size_t n, const CrcTables& T, uint32_t c = 0xFFFFFFFFu) {
  for (size_t i = 0; i < n; ++i) c = T.byte[(c ^ p[i]) & 0xffu] ^ (c >> 8);
  return c;
}

/* ---------------------------------------------------------------- PNG ---- */
constexpr uint32_t kMaxStoredBlock = 65535; /* png.zig:8 */
constexpr uint32_t kHeadBytes = 41;         /* signature 8 + IHDR chunk 25 + IDAT length 4 + "IDAT" 4 */

PngLayout png_layout(uint64_t width, uint64_t height) {
  PngLayout L;
  memset(&L, 0, sizeof L);
  const uint64_t max31 = 0x7FFFFFFFull;
  if (width == 0 || height == 0 || width > max31 || height > max31) return L; /* png.zig:12-13 */
  const uint64_t raw_len = (width * 3 + 1) * height;                          /* png.zig:29 */
  const uint64_t blocks = (raw_len + kMaxStoredBlock - 1) / kMaxStoredBlock;
  const uint64_t zlib_len = 2 + raw_len + 5 * blocks + 4;
  if (zlib_len > max31) return L; /* png.zig:32 */
  L.width = (uint32_t)width;
  L.height = (uint32_t)height;
  L.row_bytes = (uint32_t)(3 * width);
  L.raw_len = (uint32_t)raw_len;
  L.blocks = (uint32_t)blocks;
  L.zlib_len = (uint32_t)zlib_len;
  L.idat_data = kHeadBytes;
  const uint64_t total = kHeadBytes + zlib_len + 4 /* IDAT CRC */ + 12 /* IEND chunk */;
  if (total > 0xFFFFFFFFull) return PngLayout{};
  L.total = (uint32_t)total;
  return L;
}

static void put_be32(uint8_t* p, uint32_t v) {
  p[0] = (uint8_t)(v >> 24);
  p[1] = (uint8_t)(v >> 16);
  p[2] = (uint8_t)(v >> 8);
  p[3] = (uint8_t)v;
}

/* Signature, IHDR chunk, IDAT length and type (png.zig:15-38); IEND chunk. */
struct PngFrame {
  uint8_t head[kHeadBytes];
  uint8_t tail[12];
};

static PngFrame png_frame(const PngLayout& L, const CrcTables& T) {
  PngFrame F;
  static const uint8_t sig[8] = {0x89, 'P', 'N', 'G', '\r', '\n', 0x1a, '\n'};
  memcpy(F.head, sig, 8);
  uint8_t* ihdr = F.head + 8;
  put_be32(ihdr, 13);
  memcpy(ihdr + 4, "IHDR", 4);
  put_be32(ihdr + 8, L.width);
  put_be32(ihdr + 12, L.height);
  ihdr[16] = 8; /* bit depth */
  ihdr[17] = 2; /* truecolour */
  ihdr[18] = 0; /* deflate */
  ihdr[19] = 0; /* filter method */
  ihdr[20] = 0; /* no interlace */
  put_be32(ihdr + 21, ~crc32_host(ihdr + 4, 17, T));
  put_be32(F.head + 33, L.zlib_len);
  memcpy(F.head + 37, "IDAT", 4);
  put_be32(F.tail, 0);
  memcpy(F.tail + 4, "IEND", 4);
  put_be32(F.tail + 8, ~crc32_host(F.tail + 4, 4, T));
  return F;
}

/* One byte of the file at position q, except the Adler-32 and IDAT CRC
 * fields, which are left to the checksum kernels. */
__global__ void k_png_body(const uint8_t* __restrict__ rgb, PngLayout L, PngFrame F, uint8_t* __restrict__ png) {
  const uint32_t stride = gridDim.x * blockDim.x;
  const uint32_t adler_at = L.idat_data + L.zlib_len - 4, crc_at = L.idat_data + L.zlib_len;
  const uint32_t tail_at = crc_at + 4;
  for (uint32_t q = blockIdx.x * blockDim.x + threadIdx.x; q < L.total; q += stride) {
    uint8_t v;
    if (q < kHeadBytes) {
      v = F.head[q];
    } else if (q >= tail_at) {
      v = F.tail[q - tail_at];
    } else if (q >= adler_at) {
      continue; /* Adler-32 and CRC fields */
    } else {
      const uint32_t z = q - L.idat_data;
      if (z < 2) {
        v = z == 0 ? 0x78 : 0x01; /* zlib header, png.zig:40 */
      } else {
        const uint32_t r = z - 2;
        const uint32_t b = r / (kMaxStoredBlock + 5), off = r - b * (kMaxStoredBlock + 5);
        if (off < 5) { /* stored block header, png.zig:103-110 */
          const uint32_t remaining = L.raw_len - b * kMaxStoredBlock;
          const uint32_t len = remaining < kMaxStoredBlock ? remaining : kMaxStoredBlock;
          const uint32_t nlen = ~len & 0xFFFFu;
          v = off == 0 ? (uint8_t)(len == remaining ? 1 : 0)
              : off == 1 ? (uint8_t)(len & 0xFF)
              : off == 2 ? (uint8_t)(len >> 8)
              : off == 3 ? (uint8_t)(nlen & 0xFF)
                         : (uint8_t)(nlen >> 8);
        } else { /* the raw stream: a 0 filter byte, then the row (png.zig:42-46) */
          const uint32_t i = b * kMaxStoredBlock + (off - 5);
          const uint32_t y = i / (L.row_bytes + 1), c = i - y * (L.row_bytes + 1);
          v = c == 0 ? 0 : __ldg(rgb + (size_t)y * L.row_bytes + (c - 1));
        }
      }
    }
    png[q] = v;
  }
}

/* Adler-32 sums over the raw stream: acc[0] += sum d_i, acc[1] +=
 * sum (raw_len - i) d_i, each block's share reduced mod 65521.  Filter
 * bytes are zero and add nothing, so only the RGB bytes are visited. */
__global__ void k_adler(const uint8_t* __restrict__ rgb, PngLayout L, unsigned long long* __restrict__ acc) {
  const uint32_t n_rgb = L.row_bytes * L.height;
  const uint32_t stride = gridDim.x * blockDim.x;
  unsigned long long a = 0, b = 0;
  for (uint32_t j = blockIdx.x * blockDim.x + threadIdx.x; j < n_rgb; j += stride) {
    const uint32_t y = j / L.row_bytes, c = j - y * L.row_bytes;
    const uint32_t i = y * (L.row_bytes + 1) + 1 + c;
    const uint32_t d = __ldg(rgb + j);
    a += d;
    b += (unsigned long long)((L.raw_len - i) % 65521u) * d;
  }
  a %= 65521u;
  b %= 65521u;
  for (int o = 16; o > 0; o >>= 1) {
    a += __shfl_down_sync(0xffffffffu, a, o);
    b += __shfl_down_sync(0xffffffffu, b, o);
  }
  __shared__ unsigned long long sa[32], sb[32];
  const int w = threadIdx.x / 32, l = threadIdx.x % 32;
  if (l == 0) {
    sa[w] = a;
    sb[w] = b;
  }
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned long long ta = 0, tb = 0;
    for (int k = 0; k < (int)(blockDim.x + 31) / 32; ++k) {
      ta += sa[k];
      tb += sb[k];
    }
    atomicAdd(acc, ta % 65521u);
    atomicAdd(acc + 1, tb % 65521u);
  }
}

/* Writes Adler-32 (png.zig:47-50) big-endian into the zlib trailer. */
__global__ void k_adler_write(const unsigned long long* __restrict__ acc, PngLayout L, uint8_t* __restrict__ png) {
  const uint32_t A = (uint32_t)((1 + acc[0]) % 65521u);
  const uint32_t B = (uint32_t)(((unsigned long long)(L.raw_len % 65521u) + acc[1]) % 65521u);
  const uint32_t v = (B << 16) | A;
  uint8_t* p = png + L.idat_data + L.zlib_len - 4;
  p[0] = (uint8_t)(v >> 24);
  p[1] = (uint8_t)(v >> 16);
  p[2] = (uint8_t)(v >> 8);
  p[3] = (uint8_t)v;
}

static uint32_t crc_slices(const PngLayout& L) {
  const uint32_t n = 4 + L.zlib_len; /* "IDAT" + data */
  return (n + kCrcSlice - 1) / kCrcSlice;
}

size_t png_scratch_bytes(const PngLayout& L) { return 2 * sizeof(unsigned long long) + crc_slices(L) * 4; }

zt_status launch_png(const uint8_t* d_rgb, const PngLayout& L, uint8_t* d_png, void* d_scratch, cudaStream_t stream) {
  static const CrcTables T = make_crc_tables();
  const PngFrame F = png_frame(L, T);
  unsigned long long* acc = static_cast<unsigned long long*>(d_scratch);
  uint32_t* slices = reinterpret_cast<uint32_t*>(acc + 2);
  cudaError_t e = cudaMemsetAsync(acc, 0, 2 * sizeof(unsigned long long), stream);
  if (e != cudaSuccess) return out_cuda_fail(e, "png: clear Adler-32 sums");
  k_png_body<<<stride_grid(L.total, 256), 256, 0, stream>>>(d_rgb, L, F, d_png);
  k_adler<<<stride_grid((uint64_t)L.row_bytes * L.height, 256), 256, 0, stream>>>(d_rgb, L, acc);
  k_adler_write<<<1, 1, 0, stream>>>(acc, L, d_png);
  const uint32_t n = 4 + L.zlib_len, ns = crc_slices(L);
  k_crc_blocks<<<ns, kCrcThreads, 0, stream>>>(d_png + L.idat_data - 4, n, T, slices);
  k_crc_final<<<1, kCrcThreads, 0, stream>>>(slices, ns, n, T, d_png + L.idat_data + L.zlib_len);
  e = cudaGetLastError();
  return e == cudaSuccess ? ZT_OK : out_cuda_fail(e, "launch png kernels");
}

/* png.writePng on the host, sequentially (the same bytes). */
static void png_host(const uint8_t* rgb, const PngLayout& L, uint8_t* out) {
  static const CrcTables T = make_crc_tables();
  const PngFrame F = png_frame(L, T);
  memcpy(out, F.head, kHeadBytes);
  uint8_t* z = out + L.idat_data;
  size_t w = 0;
  z[w++] = 0x78;
  z[w++] = 0x01;
  uint32_t remaining = L.raw_len, block_left = 0, a = 1, b = 0;
  auto put = [&](uint8_t byte) {
    if (block_left == 0) { /* StoredDeflate.startBlock, png.zig:103-111 */
      const uint32_t len = remaining < kMaxStoredBlock ? remaining : kMaxStoredBlock;
      z[w++] = (uint8_t)(len == remaining ? 1 : 0);
      z[w++] = (uint8_t)(len & 0xFF);
      z[w++] = (uint8_t)(len >> 8);
      z[w++] = (uint8_t)(~len & 0xFF);
      z[w++] = (uint8_t)((~len >> 8) & 0xFF);
      block_left = len;
    }
    z[w++] = byte;
    a = (a + byte) % 65521u;
    b = (b + a) % 65521u;
    --block_left;
    --remaining;
  };
  for (uint32_t y = 0; y < L.height; ++y) {
    put(0);
    for (uint32_t c = 0; c < L.row_bytes; ++c) put(rgb[(size_t)y * L.row_bytes + c]);
  }
  put_be32(z + w, (b << 16) | a);
  w += 4;
  put_be32(z + w, ~crc32_host(out + L.idat_data - 4, 4 + L.zlib_len, T));
  memcpy(z + w + 4, F.tail, 12);
}

}  // namespace zt

using namespace zt;

extern "C" {

zt_status zt_png_size(uint64_t width, uint64_t height, uint64_t* bytes_out) {
  if (!bytes_out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_png_size: NULL output");
  const PngLayout L = png_layout(width, height);
  *bytes_out = L.total;
  if (L.total == 0) {
    if (width == 0 || height == 0 || width > 0x7FFFFFFFull || height > 0x7FFFFFFFull)
      return fail(ZT_ERR_INVALID_ARGUMENT, "InvalidDimensions: width and height must be in 1 .. 2^31-1");
    return fail(ZT_ERR_INVALID_ARGUMENT, "ImageTooLarge: the zlib stream would exceed 2^31-1 bytes");
  }
  return ZT_OK;
}

zt_status zt_png_encode(const uint8_t* rgb, uint64_t width, uint64_t height, uint8_t* out, uint64_t out_capacity) {
  uint64_t need = 0;
  const zt_status rc = zt_png_size(width, height, &need);
  if (rc != ZT_OK) return rc;
  if (!rgb || !out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_png_encode: NULL argument");
  if (out_capacity < need) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_png_encode: output smaller than zt_png_size");
  png_host(rgb, png_layout(width, height), out);
  return ZT_OK;
}

zt_status zt_png_encode_device(const uint8_t* d_rgb, uint64_t width, uint64_t height, uint8_t* d_out,
                               uint64_t out_capacity, void* stream) {
  uint64_t need = 0;
  const zt_status rc = zt_png_size(width, height, &need);
  if (rc != ZT_OK) return rc;
  if (!d_rgb || !d_out) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_png_encode_device: NULL argument");
  if (out_capacity < need) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_png_encode_device: output smaller than zt_png_size");
  const PngLayout L = png_layout(width, height);
  cudaStream_t s = (cudaStream_t)stream;
  void* scratch = nullptr;
  cudaError_t e = cudaMallocAsync(&scratch, png_scratch_bytes(L), s);
  if (e != cudaSuccess) return out_cuda_fail(e, "zt_png_encode_device: scratch");
  const zt_status r = launch_png(d_rgb, L, d_out, scratch, s);
  e = cudaFreeAsync(scratch, s);
  if (r != ZT_OK) return r;
  return e == cudaSuccess ? ZT_OK : out_cuda_fail(e, "zt_png_encode_device: free scratch");
}

zt_status zt_image_to_rgb8_device(const double* d_pixels, uint64_t n_pixels, uint32_t tonemap, double gamma,
                                  double exposure, uint8_t* d_rgb_out, void* stream) {
  if ((!d_pixels || !d_rgb_out) && n_pixels) return fail(ZT_ERR_INVALID_ARGUMENT, "zt_image_to_rgb8_device: NULL argument");
  if (tonemap > 2) return fail(ZT_ERR_INVALID_ARGUMENT, "tonemap must be 0 (none), 1 (reinhard) or 2 (aces)");
  return launch_encode_rgb8(d_pixels, 3 * n_pixels, tonemap, gamma, exposure, d_rgb_out, (cudaStream_t)stream);
}

}  /* extern "C" */
