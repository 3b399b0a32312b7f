/*
 * output.cuh -- device side of the output stage (src/image.zig:14-73,
 * src/png.zig:10-117): 8-bit encode of the HDR framebuffer and the PNG
 * stream assembled on the device.  Launchers used by render.cu's
 * render-to-PNG entry points; the C-ABI functions live in output.cu.
 */
#ifndef ZT_OUTPUT_CUH
#define ZT_OUTPUT_CUH

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/zigtrace_b200.h"

namespace zt {

/* Byte layout of the PNG that png.zig:10-58 writes for a w x h RGB8 image.
 * total == 0 marks dimensions the reference rejects (zero, above 2^31 - 1,
 * or a zlib stream longer than 2^31 - 1 bytes). */
struct PngLayout {
  uint32_t width, height;
  uint32_t row_bytes;   /* 3 * width */
  uint32_t raw_len;     /* (3 * width + 1) * height: rows with their filter byte */
  uint32_t blocks;      /* stored DEFLATE blocks of at most 65535 bytes */
  uint32_t zlib_len;    /* 2 + raw_len + 5 * blocks + 4 */
  uint32_t idat_data;   /* offset of the zlib stream in the file */
  uint32_t total;       /* file length */
};

PngLayout png_layout(uint64_t width, uint64_t height);

/* Encodes n_values f64 channel values to u8 on `stream` (Output.encode). */
zt_status launch_encode_rgb8(const double* d_px, uint64_t n_values, uint32_t tonemap, double gamma, double exposure,
                             uint8_t* d_out, cudaStream_t stream);

/* Writes the whole PNG file for d_rgb (L.width x L.height x 3 bytes) into
 * d_png (L.total bytes) on `stream`.  d_scratch: png_scratch_bytes(L)
 * bytes of device memory. */
size_t png_scratch_bytes(const PngLayout& L);
zt_status launch_png(const uint8_t* d_rgb, const PngLayout& L, uint8_t* d_png, void* d_scratch, cudaStream_t stream);

}  // namespace zt

#endif
