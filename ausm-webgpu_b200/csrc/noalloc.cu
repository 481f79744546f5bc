// ausm_forces_noalloc: the surface force and wall pressure coefficients of a state the
// caller already holds in device memory, computed without allocating anything.
//
// It is for hosts that cannot call cudaMalloc at the point where they need the forces:
// a host that owns every device buffer through its own pool or arena (and forbids
// allocations made behind its back), a host that runs this between launches it has
// already laid out and must not trigger the implicit synchronisation an allocation can
// cause, or a host that has no solver handle at all because the state lives in its own
// buffers.  Such a caller passes device pointers to its data and host pointers for the
// results; the library uses only the fixed scratch array below.
//
// Scratch: g_noalloc_scratch, a file-scope __device__ array of 3 * kNoAllocMaxFaces + 2
// doubles (384 KiB + 16 B) holding, per wall face, the force (x, y) and Cp, then the two
// summed force components.  Every GPU that loads the library holds one copy until the
// process exits.  Host code never uses the array's name as an address: on the first
// call on each device (with that device current) cudaGetSymbolAddress gives the device
// address, which is cached per device and passed to the kernels.  Because that first
// call performs this set-up, it should come before any stream capture.  All calls on a
// device share the one array and it keeps the last call's contents; every slot a call
// reads is written earlier in the same call, so nothing needs clearing, but two calls
// whose kernels overlap on the GPU (different streams, or host threads) race on it.
#include <cmath>
#include <mutex>
#include <string>

#include "ausm.h"
#include "ausm_internal.h"

namespace ausm {
void set_thread_error(const std::string& msg);  // api.cu
}

namespace {

constexpr int kNoAllocMaxFaces = 16384;
constexpr int kScratchDoubles = 3 * kNoAllocMaxFaces + 2;
constexpr int kMaxDevices = 64;

__device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

std::mutex g_scratch_mu;
double* g_scratch_ptr[kMaxDevices] = {};

// Per wall face i (vertices i, i+1 of row 0): f32 pressure of the first interior cell
// as the reference computes it (graphs.js:26-39), FP64 length, inward normal force
// -p l n and Cp = (p - p_inf) / q_inf.
__global__ void k_face_forces_noalloc(const float4* __restrict__ row0, const float2* __restrict__ body, int M,
                                      float gamma, double q_inf, double p_inf, double* __restrict__ scratch) {
  for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < M; i += gridDim.x * blockDim.x) {
    float4 s = row0[i];
    float rho = s.x, u = s.y / rho, v = s.z / rho;
    float p = (s.w - 0.5f * rho * (u * u + v * v)) * (gamma - 1.0f);
    float2 a = body[i], b = body[i + 1 == M ? 0 : i + 1];
    double dx = (double)b.x - a.x, dy = (double)b.y - a.y;
    double len = sqrt(dx * dx + dy * dy);
    double nx = dy / len, ny = -dx / len;
    scratch[i] = -(double)p * len * nx;
    scratch[kNoAllocMaxFaces + i] = -(double)p * len * ny;
    scratch[2 * kNoAllocMaxFaces + i] = ((double)p - p_inf) / q_inf;
  }
}

// One block of 256 threads: fixed-order strided partial sums, then a tree, into the
// two result slots (deterministic).
__global__ void k_sum_forces_noalloc(int M, double* __restrict__ scratch) {
  __shared__ double sx[256], sy[256];
  const int t = threadIdx.x;
  double ax = 0.0, ay = 0.0;
  for (int i = t; i < M; i += 256) {
    ax += scratch[i];
    ay += scratch[kNoAllocMaxFaces + i];
  }
  sx[t] = ax;
  sy[t] = ay;
  __syncthreads();
  for (int s = 128; s > 0; s >>= 1) {
    if (t < s) {
      sx[t] += sx[t + s];
      sy[t] += sy[t + s];
    }
    __syncthreads();
  }
  if (t == 0) {
    scratch[3 * kNoAllocMaxFaces] = sx[0];
    scratch[3 * kNoAllocMaxFaces + 1] = sy[0];
  }
}

int fail_na(int code, const std::string& msg) {
  ausm::set_thread_error(msg);
  return code;
}

}  // namespace

extern "C" int ausm_forces_noalloc(const void* wall_row, const void* body_xy, int M, const AusmParams* p,
                                   double* out6, double* cp, void* stream) {
  if (!wall_row || !body_xy || !p || !out6) return fail_na(AUSM_ERR_INVALID, "null argument");
  if (M < 4) return fail_na(AUSM_ERR_INVALID, "M must be >= 4");
  if (M > kNoAllocMaxFaces)
    return fail_na(AUSM_ERR_INVALID, "M = " + std::to_string(M) + " exceeds the no-allocation scratch limit of " +
                                         std::to_string(kNoAllocMaxFaces) + " wall faces");
  if (!(p->gamma > 1.0 && p->in_rho > 0.0 && p->in_pressure > 0.0 && p->mach > 0.0))
    return fail_na(AUSM_ERR_INVALID, "need gamma > 1, in_rho > 0, in_pressure > 0 and mach > 0");
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return fail_na(AUSM_ERR_CUDA, std::string("cudaGetDevice: ") + cudaGetErrorString(e));
  if (dev < 0 || dev >= kMaxDevices)
    return fail_na(AUSM_ERR_INVALID, "device index " + std::to_string(dev) + " is above the " +
                                         std::to_string(kMaxDevices) + " devices this entry point serves");
  double* scratch = nullptr;
  {
    std::lock_guard<std::mutex> lock(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {  // once per device, with that device current
      void* ptr = nullptr;
      e = cudaGetSymbolAddress(&ptr, g_noalloc_scratch);
      if (e != cudaSuccess || !ptr)
        return fail_na(AUSM_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
      g_scratch_ptr[dev] = static_cast<double*>(ptr);
    }
    scratch = g_scratch_ptr[dev];
  }
  cudaStream_t s = static_cast<cudaStream_t>(stream);
  const double a = p->aoa_deg * M_PI / 180.0;
  const double speed = p->mach * std::sqrt(p->gamma * p->in_pressure / p->in_rho);
  const double vx = speed * std::cos(a), vy = speed * std::sin(a);
  const double q_inf = 0.5 * p->in_rho * (vx * vx + vy * vy);
  k_face_forces_noalloc<<<(M + 255) / 256, 256, 0, s>>>(static_cast<const float4*>(wall_row),
                                                        static_cast<const float2*>(body_xy), M, (float)p->gamma, q_inf,
                                                        p->in_pressure, scratch);
  k_sum_forces_noalloc<<<1, 256, 0, s>>>(M, scratch);
  e = cudaGetLastError();
  if (e != cudaSuccess) return fail_na(AUSM_ERR_CUDA, std::string("launch: ") + cudaGetErrorString(e));
  double F[2];
  e = cudaMemcpyAsync(F, scratch + 3 * kNoAllocMaxFaces, 2 * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess && cp)
    e = cudaMemcpyAsync(cp, scratch + 2 * kNoAllocMaxFaces, (size_t)M * sizeof(double), cudaMemcpyDeviceToHost, s);
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess) return fail_na(AUSM_ERR_CUDA, std::string("copy-out: ") + cudaGetErrorString(e));
  const double nx = vx / speed, ny = vy / speed, invQ = 1.0 / q_inf;
  const double Cl = (F[0] * -ny + F[1] * nx) * invQ, Cd = (F[0] * nx + F[1] * ny) * invQ;
  const double FV = F[0] * nx + F[1] * ny;
  out6[0] = F[0];
  out6[1] = F[1];
  out6[2] = std::sqrt(F[0] * F[0] + F[1] * F[1]) * (FV > 0 ? 1.0 : (FV < 0 ? -1.0 : 0.0));
  out6[3] = Cl;
  out6[4] = Cd;
  out6[5] = Cl / Cd;
  return AUSM_OK;
}
