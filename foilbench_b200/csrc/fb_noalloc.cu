// Allocation-free variant of the Jacobi viscosity operator (fb_op_implicit_diffuse).
//
// Some hosts of this library cannot let it allocate device memory: a simulation or viewer
// loop that owns every device byte through its own pool (sized once at start-up) and forbids
// driver allocations while it runs, because a cudaMalloc there would exceed its budget or
// stall its frame on the driver's implicit synchronisation. This entry point takes the
// caller's device buffers for input and output and keeps its working set (Jacobi ping-pong
// planes, reduction partials, barrier and report words) in one file-scope device array of
// fixed size, so it never calls cudaMalloc, cudaFree or any allocating routine.
//
// The array is shared by every call on a device and keeps the previous call's contents;
// the barrier and report words are cleared at the start of each call. Calls whose work
// overlaps on the GPU (for example issued to different streams) race on the array. A call
// returns after its kernel has finished: it waits on the stream and reads the report back.

#include <algorithm>
#include <cstdio>
#include <cstring>
#include <mutex>

#include <cuda_runtime.h>

#include "../../include/foilb200.h"
#include "fb_step.cuh"

namespace fb {
void *step_kernel_f64(int vpt, int r0);
void *step_kernel_f32r(int vpt, int r0);
void set_last_error(const char *message);                 // fb_last_error() text (fb_lib.cu)
void fill_report(const DevReport &r, fb_report *out);     // device report -> fb_report (fb_lib.cu)
}  // namespace fb

using namespace fb;

namespace {

constexpr size_t kScratchBytes = (size_t)FB_NOALLOC_SCRATCH_BYTES;
constexpr int kThreadsNA = 512;
constexpr int kMaxDevices = 64;
constexpr int kMaxBlocks = 2048;

static __device__ __align__(256) unsigned char g_scratch[kScratchBytes];

std::mutex g_mu;
char *g_base[kMaxDevices] = {};  // device address of g_scratch per device (set up once)

thread_local char g_msg[512];

int err(int code, const char *msg) {
  std::snprintf(g_msg, sizeof(g_msg), "%s", msg);
  fb::set_last_error(g_msg);
  return code;
}

size_t up256(size_t n) { return (n + 255) / 256 * 256; }

// Makes `device` current for the call and gives the caller's current device back on every
// return path, so a host that manages several devices keeps its own runtime state.
struct DeviceGuard {
  int prev = -1;
  bool ok = false;
  explicit DeviceGuard(int device) {
    ok = cudaGetDevice(&prev) == cudaSuccess && cudaSetDevice(device) == cudaSuccess;
  }
  ~DeviceGuard() {
    if (prev >= 0) cudaSetDevice(prev);
  }
};

}  // namespace

extern "C" {

int32_t fb_op_implicit_diffuse_noalloc(int32_t device, const fb_scenario_desc *desc, const void *vx_in,
                                       const void *vy_in, void *vx_out, void *vy_out, double viscosity, double dt,
                                       double tolerance, int32_t max_iterations, void *stream, fb_report *out) {
  if (!desc || !vx_in || !vy_in || !vx_out || !vy_out) return err(FB_ERR_INVALID_ARGUMENT, "null argument");
  if (desc->nx < 4 || desc->ny < 4) return err(FB_ERR_INVALID_ARGUMENT, "each resolution axis must contain at least four cells");
  if (desc->precision != FB_FLOAT32 && desc->precision != FB_FLOAT64) return err(FB_ERR_INVALID_ARGUMENT, "precision");
  if (!(desc->x1 > desc->x0) || !(desc->y1 > desc->y0)) return err(FB_ERR_INVALID_ARGUMENT, "invalid bounds");
  if (device < 0 || device >= kMaxDevices) return err(FB_ERR_INVALID_ARGUMENT, "device index out of range");
  const size_t n = (size_t)desc->nx * desc->ny;
  const size_t vsz = desc->precision == FB_FLOAT64 ? 8 : 4;
  const size_t plane = up256(n * vsz);
  const size_t part_off = 4 * plane;
  const size_t gs_off = up256(part_off + (size_t)SL_COUNT * kMaxBlocks * sizeof(double));
  const size_t rep_off = up256(gs_off + sizeof(GridSync));
  const size_t need = up256(rep_off + sizeof(DevReport));
  if (need > kScratchBytes) {
    // largest grid: four 256-byte-rounded planes beside the fixed header (partials, barrier,
    // report), i.e. 2,084,832 cells in float64 and 4,169,664 in float32
    const size_t max_plane = (kScratchBytes - (need - 4 * plane)) / 4 / 256 * 256;
    std::snprintf(g_msg, sizeof(g_msg),
                  "grid %dx%d needs %zu bytes of scratch; the allocation-free entry point holds %zu "
                  "(at most %zu cells in this precision)",
                  desc->nx, desc->ny, need, kScratchBytes, max_plane / vsz);
    fb::set_last_error(g_msg);
    return FB_ERR_INVALID_ARGUMENT;
  }
  DeviceGuard guard(device);
  if (!guard.ok) return err(FB_ERR_CUDA, "cudaSetDevice failed");
  char *base = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_mu);
    if (!g_base[device]) {
      // one-time set-up on this device (with it current): the host-side name of the array is
      // not a device address, so ask the runtime for the device address once and keep it
      void *p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_scratch);
      if (e != cudaSuccess) {
        std::snprintf(g_msg, sizeof(g_msg), "cudaGetSymbolAddress: %s", cudaGetErrorString(e));
        fb::set_last_error(g_msg);
        return FB_ERR_CUDA;
      }
      g_base[device] = static_cast<char *>(p);
    }
    base = g_base[device];
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  void *kernel = desc->precision == FB_FLOAT64 ? step_kernel_f64(8, 8) : step_kernel_f32r(8, 8);
  int occ = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kernel, kThreadsNA, 0) != cudaSuccess || occ < 1)
    return err(FB_ERR_CUDA, "occupancy query failed");
  if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device) != cudaSuccess)
    return err(FB_ERR_CUDA, "device attribute query failed");
  long long want = (long long)((n + 2 * kThreadsNA - 1) / (2 * kThreadsNA));
  int nblocks = (int)std::min<long long>(std::min<long long>((long long)occ * sms, want), kMaxBlocks);
  if (nblocks < 1) nblocks = 1;
  // clear what must start at zero: barrier state and report
  if (cudaMemsetAsync(base + gs_off, 0, rep_off + sizeof(DevReport) - gs_off, st) != cudaSuccess)
    return err(FB_ERR_CUDA, "clearing the scratch header failed");

  auto fill = [&](auto tag) -> int {
    using V = decltype(tag);
    StepParams<V, double> p{};
    p.nx = desc->nx;
    p.ny = desc->ny;
    auto axis = [](double lo, double hi, int nn, int per) {
      Axis a{};
      a.lo = lo;
      a.hi = hi;
      a.h = (hi - lo) / nn;
      a.start = lo + 0.5 * a.h;
      a.stop = hi - 0.5 * a.h;
      a.step = (a.stop - a.start) / (double)(nn - 1);
      a.n = nn;
      a.periodic = per;
      return a;
    };
    p.ax = axis(desc->x0, desc->x1, desc->nx, desc->periodic_x);
    p.ay = axis(desc->y0, desc->y1, desc->ny, desc->periodic_y);
    p.phases = PH_DIFFUSE | PH_CELLS_ONLY;
    p.dt = dt;
    p.nu = viscosity;
    p.vtol = tolerance;
    p.vmaxit = max_iterations;
    p.cx = const_cast<V *>(static_cast<const V *>(vx_in));
    p.cy = const_cast<V *>(static_cast<const V *>(vy_in));
    p.fx = reinterpret_cast<V *>(base);
    p.gx = reinterpret_cast<V *>(base + plane);
    p.fy = reinterpret_cast<V *>(base + 2 * plane);
    p.gy = reinterpret_cast<V *>(base + 3 * plane);
    p.hx = static_cast<V *>(vx_out);
    p.hy = static_cast<V *>(vy_out);
    p.part = reinterpret_cast<double *>(base + part_off);
    p.gs = reinterpret_cast<GridSync *>(base + gs_off);
    p.rep = reinterpret_cast<DevReport *>(base + rep_off);
    p.limit_ns = 2000000000ull;
    void *args[] = {&p};
    const cudaError_t e = cudaLaunchCooperativeKernel(kernel, dim3(nblocks), dim3(kThreadsNA), args, 0, st);
    if (e != cudaSuccess) {
      std::snprintf(g_msg, sizeof(g_msg), "launch: %s", cudaGetErrorString(e));
      fb::set_last_error(g_msg);
      return FB_ERR_CUDA;
    }
    return FB_OK;
  };
  const int rc = desc->precision == FB_FLOAT64 ? fill(0.0) : fill(0.0f);
  if (rc) return rc;
  DevReport rep;
  std::memset(&rep, 0, sizeof(rep));
  if (cudaMemcpyAsync(&rep, base + rep_off, sizeof(rep), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return err(FB_ERR_CUDA, "reading the report failed");
  if (out) {
    std::memset(out, 0, sizeof(*out));
    fb::fill_report(rep, out);  // same status mapping as fb_op_implicit_diffuse
    out->kernel_launches = 1;
  }
  if (rep.status == ST_TIMEOUT) return err(FB_ERR_DEVICE_TIMEOUT, "device barrier wait timed out");
  if (rep.status != ST_OK) {
    std::snprintf(g_msg, sizeof(g_msg), "numerical failure reason=%d stage=%d", rep.reason, rep.stage);
    fb::set_last_error(g_msg);
    return FB_ERR_NUMERICAL;
  }
  return FB_OK;
}

}  // extern "C"
