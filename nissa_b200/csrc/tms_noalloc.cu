// Allocation-free e/o hopping: tms_hop_eo_noalloc.
//
// Some callers cannot let a library call cudaMalloc/cudaFree: an application
// whose device memory is all handed out by its own caching pool (as nissa's
// memory manager does, base/memory_manager.hpp) and that must not see memory
// appear behind its back, or code in a phase where an allocation or a free
// would force a device-wide synchronisation.  This entry point serves them: it
// runs the same hopping kernel as tms_hop_eo, on the caller's device buffers,
// and keeps its scratch (the structure-of-arrays copies of the links and of
// the input/output spinors) in one fixed device array declared below.
//
// The array is a file-scope __device__ variable of TMS_NOALLOC_MAX_SITES * 768
// + 256 bytes (12 MiB): every GPU that loads this library holds it until the
// process exits.  With CUDA's lazy module loading (the default) the library's
// device code, and with it this array, is loaded onto a device the first time
// it is needed there; the first call of tms_hop_eo_noalloc on a device does
// that (its cudaGetSymbolAddress set-up forces the load), so that call is the
// one that makes the 12 MiB appear and may synchronise: make it outside any
// phase that must not see either.  Every call shares the array and it keeps
// the last call's contents; calls whose work overlaps on the GPU (two streams,
// two host threads) race on it and must be serialised by the caller.  Each
// call writes every scratch element before reading it, so nothing has to
// start at zero.  The device address found at set-up is kept per device
// ordinal for the life of the process; after cudaDeviceReset the module is
// reloaded and may sit elsewhere, so this entry point is not for use across a
// device reset.
#include "tmsolve.h"
#include "tms_kernels.cuh"

#include <cstdio>
#include <mutex>

using namespace tms;

namespace
{
  constexpr int64_t kMaxSites = TMS_NOALLOC_MAX_SITES;
  // links: V x 4 x 9 double2 (576 B per site); spinors in + out: 2 x Vh x 12 double2 (192 B per site)
  constexpr size_t kLinkBytes = (size_t)kMaxSites * 576;
  // + one 256-byte slot for the operator parameters
  constexpr size_t kScratchBytes = (size_t)kMaxSites * 768 + 256;

  static __device__ __align__(256) unsigned char noalloc_scratch[kScratchBytes];

  constexpr int kMaxDevices = 64;
  std::mutex setup_mutex;
  void* scratch_addr[kMaxDevices] = {nullptr};

  void set_err(char* err, int errlen, const char* msg)
  {
    if (err && errlen > 0) snprintf(err, (size_t)errlen, "%s", msg);
  }

  // Host code must not use noalloc_scratch as an address (it names a host-side
  // stand-in): look up the device address once per device, with it current.
  tms_status scratch_for_current_device(void** out, char* err, int errlen)
  {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices)
      {
        set_err(err, errlen, "tms_hop_eo_noalloc: no usable current CUDA device");
        return TMS_ERR_CUDA;
      }
    std::lock_guard<std::mutex> lock(setup_mutex);
    if (!scratch_addr[dev])
      {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, noalloc_scratch);
        if (e != cudaSuccess || !p)
          {
            char buf[256];
            snprintf(buf, sizeof buf, "tms_hop_eo_noalloc: cudaGetSymbolAddress failed: %s", cudaGetErrorString(e));
            set_err(err, errlen, buf);
            return TMS_ERR_CUDA;
          }
        scratch_addr[dev] = p;
      }
    *out = scratch_addr[dev];
    return TMS_OK;
  }

  // AoS conf (lx or e/o layout) -> SoA e/o links, lx index computed from the site
  __global__ void noalloc_conf_kernel(Lattice g, const double* __restrict__ src, int layout, int unfold,
                                      double2* __restrict__ U)
  {
    const int idx = blockIdx.x * blockDim.x + threadIdx.x;
    if (idx >= g.V) return;
    const int p = idx >= g.Vh, ieo = idx - (p ? (int)g.Vh : 0);
    const Site s = eo_site(g, p, ieo);
    const size_t row = (layout == TMS_LAYOUT_LX) ? (size_t)s.lx : (size_t)idx;
    const double* a = src + row * 72; // 8-byte accesses: the caller's buffer need not be 16-byte aligned
    for (int mu = 0; mu < 4; mu++)
      {
        const double sg = (unfold && mu == 0 && s.t == g.T - 1) ? g.bc_t : 1.0;
        for (int k = 0; k < 9; k++)
          {
            const double wx = a[2 * (mu * 9 + k)], wy = a[2 * (mu * 9 + k) + 1];
            U[((size_t)(p * 4 + mu) * 9 + k) * g.Vh + ieo] = make_double2(wx * sg, wy * sg);
          }
      }
  }
}

extern "C" tms_status tms_hop_eo_noalloc(int T, int L, double bc_t, const double* conf, int layout, int flags,
                                         int par_out, const double* in, double* out, int has_anis, double anis,
                                         void* stream, char* err, int errlen)
{
  set_err(err, errlen, "");
  if (T <= 0 || L <= 0 || (T & 1) || (L & 1) || !conf || !in || !out || (par_out != 0 && par_out != 1) ||
      (layout != TMS_LAYOUT_LX && layout != TMS_LAYOUT_EO))
    {
      set_err(err, errlen, "tms_hop_eo_noalloc: bad arguments (T, L even and positive; parity 0/1; non-null buffers)");
      return TMS_ERR_BAD_ARG;
    }
  const int64_t V = (int64_t)T * L * L * L;
  if (V > kMaxSites)
    {
      char buf[256];
      snprintf(buf, sizeof buf, "tms_hop_eo_noalloc: lattice of %lld sites exceeds the fixed scratch limit of %lld sites",
               (long long)V, (long long)kMaxSites);
      set_err(err, errlen, buf);
      return TMS_ERR_BAD_ARG;
    }
  void* base = nullptr;
  const tms_status st = scratch_for_current_device(&base, err, errlen);
  if (st != TMS_OK) return st;

  Lattice g;
  g.T = T;
  g.LX = g.LY = g.LZ = L;
  g.V = V;
  g.Vh = V / 2;
  g.stride = (int)g.Vh;
  g.bc_t = bc_t;
  const int n = (int)g.Vh;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  double2* U = reinterpret_cast<double2*>(base);
  unsigned char* sp = reinterpret_cast<unsigned char*>(base) + kLinkBytes;
  SpinorT<PREC_F64> sin, sout;
  sin.d = reinterpret_cast<double2*>(sp);
  sin.n = nullptr;
  sin.stride = n;
  sout.d = reinterpret_cast<double2*>(sp + (size_t)n * 192);
  sout.n = nullptr;
  sout.stride = n;

  // the operator's scalar (anisotropy) lives in the scratch too: no allocation
  OpParams* prm = reinterpret_cast<OpParams*>(sp + (size_t)n * 384);
  static_assert(sizeof(OpParams) <= 64, "OpParams slot");
  const OpParams h{1.0, 0.0, has_anis ? anis : 1.0};
  cudaError_t e = cudaMemcpyAsync(prm, &h, sizeof h, cudaMemcpyHostToDevice, s);

  if (e == cudaSuccess)
    {
      noalloc_conf_kernel<<<(int)((V + 127) / 128), 128, 0, s>>>(g, conf, layout,
                                                                   (flags & TMS_CONF_BC_INCLUDED) ? 1 : 0, U);
      aos_to_soa_kernel<PREC_F64><<<(n + 255) / 256, 256, 0, s>>>(n, in, nullptr, sin);
      EpiPlain<PREC_F64> epi{{sout, sout}};
      Reducer red{nullptr, nullptr, nullptr};
      hop_kernel<PREC_F64, LINK_F64_18, EpiPlain<PREC_F64>, NoFin><<<(n + HOP_THREADS - 1) / HOP_THREADS,
                                                                      HOP_THREADS, 0, s>>>(
        g, par_out, 1, sin, sin, LinkT<LINK_F64_18>{U, n}, prm, epi, red, NoFin{}, nullptr);
      soa_to_aos_kernel<PREC_F64><<<(n + 255) / 256, 256, 0, s>>>(n, sout, nullptr, out);
      e = cudaGetLastError();
    }
  if (e == cudaSuccess) e = cudaStreamSynchronize(s);
  if (e != cudaSuccess)
    {
      char buf[256];
      snprintf(buf, sizeof buf, "tms_hop_eo_noalloc: %s", cudaGetErrorString(e));
      set_err(err, errlen, buf);
      return TMS_ERR_CUDA;
    }
  return TMS_OK;
}
