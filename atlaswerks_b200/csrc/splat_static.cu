// splat_static.cu — a splat entry point that allocates no device memory.
//
// aw_splat() takes its bucket scratch from the stream-ordered allocator.
// Some callers must not allocate at call time: a host application that owns
// all device memory through its own pool and gives each library a fixed
// budget at start-up, or a latency-critical loop where an allocation could
// block or fail in the middle of a stream of work. aw_splat_static() serves
// them from a fixed array compiled into the library instead. The caller
// still passes the input image, the deformation and the output image.
#include <cstring>
#include <mutex>
#include <string>

#include "../../include/aw_b200.h"
#include "capi_error.h"
#include "splat.cuh"

namespace {

// Scratch for one splat: bucket offsets, cursors, source order and scan
// partials (aw::splat_scratch_bytes). Every device that loads the library
// keeps this array resident until the process exits.
static __device__ __align__(256) unsigned char g_splat_scratch[AW_SPLAT_STATIC_MAX_BYTES];

constexpr int kMaxDevices = 64;
std::mutex g_mu;
void *g_scratch_addr[kMaxDevices] = {nullptr};

int fail_static(const std::string &m) {
  aw::set_last_error(m);
  return 1;
}

// Device address of g_splat_scratch on the current device. In host code the
// array's name is only a host-side stand-in, so the address is looked up
// once per device, with that device current, and cached.
int scratch_address(void **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_static(std::string("aw_splat_static: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices) return fail_static("aw_splat_static: device index out of range");
  std::lock_guard<std::mutex> lock(g_mu);
  if (!g_scratch_addr[dev]) {
    void *p = nullptr;
    e = cudaGetSymbolAddress(&p, g_splat_scratch);
    if (e != cudaSuccess)
      return fail_static(std::string("aw_splat_static: cudaGetSymbolAddress failed: ") +
                         cudaGetErrorString(e));
    g_scratch_addr[dev] = p;
  }
  *out = g_scratch_addr[dev];
  return 0;
}

}  // namespace

extern "C" {

int aw_splat_static_fits(int nx, int ny, int nz) {
  if (nx < 1 || ny < 1 || nz < 1) return 0;
  return aw::splat_scratch_bytes(aw::Dims{nx, ny, nz}, false) <=
                 (size_t)AW_SPLAT_STATIC_MAX_BYTES
             ? 1
             : 0;
}

int aw_splat_static(const float *img, const float *hx, const float *hy, const float *hz,
                    float *out, int nx, int ny, int nz, float background, void *stream) {
  if (!img || !hx || !hy || !hz || !out) return fail_static("aw_splat_static: null pointer");
  if (nx < 1 || ny < 1 || nz < 1) return fail_static("aw_splat_static: empty grid");
  const aw::Dims d{nx, ny, nz};
  const size_t need = aw::splat_scratch_bytes(d, false);
  if (need > (size_t)AW_SPLAT_STATIC_MAX_BYTES)
    return fail_static("aw_splat_static: grid needs " + std::to_string(need) +
                       " bytes of scratch, more than the fixed " +
                       std::to_string((size_t)AW_SPLAT_STATIC_MAX_BYTES) +
                       " bytes of this entry point; use aw_splat for larger grids");
  void *scratch = nullptr;
  if (scratch_address(&scratch)) return 1;
  aw::SplatWork w;
  aw::splat_work_bind(&w, d, scratch, false);
  // aw::splat zeroes the bucket counters itself; nothing from the previous
  // call's contents is read before it is rewritten
  const cudaError_t e =
      aw::splat(w, img, hx, hy, hz, out, background, reinterpret_cast<cudaStream_t>(stream));
  if (e != cudaSuccess)
    return fail_static(std::string("aw_splat_static: ") + cudaGetErrorString(e));
  return 0;
}

}  // extern "C"
