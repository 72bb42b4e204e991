// Net-flux evaluation that allocates no device memory (cfd_evaluate_net_flux_noalloc).
//
// Some callers cannot let this library call cudaMalloc: a host code that hands all of the GPU's
// memory to its own pool allocator up front (a framework's caching allocator, a fixed-budget
// embedded solver), or a time-critical loop in which the implicit device synchronisation and the
// possible failure of a fresh cudaMalloc are not acceptable.  For them this entry point runs the
// residual kernel on arrays the caller already owns.  The only scratch the kernel needs — the
// control block that receives Min_dt, the completion counter of the last-block reduction and one
// partial minimum per thread block — lives in the file-scope device array below, of fixed size,
// which every GPU that loads the library holds until the process exits.
//
// The array is placed on a device when the library's device code is loaded into the caller's
// CUDA context.  With lazy module loading (the CUDA default since 12.2) that happens during the
// first call in a context: that call may itself need the array's 2 MiB of free device memory and
// synchronises the device.  So a caller whose pool reserves the GPU's memory makes its first
// call before the pool takes it, or sets CUDA_MODULE_LOADING=EAGER; and makes it before any
// stream capture.
#include <cuda_runtime.h>

#include <string>

#include "../../include/cfd_b200.h"
#include "kernels.cuh"

namespace {

constexpr int kMaxCells = 8388608;   // largest mesh (physical cells) one call accepts
constexpr int kMaxBlocks = 262144;   // partial-minimum slots: one per flux-kernel thread block
constexpr int kCtlDoubles = cfdb::CTL_SIZE;
constexpr int kCounterDoubles = 8;  // completion counter (unsigned) + status words (2 x int)
constexpr int kScratchDoubles = kCtlDoubles + kCounterDoubles + kMaxBlocks;

// Shared by every call on a device: a call overwrites what the previous one left.
static __device__ __align__(256) double g_noalloc_scratch[kScratchDoubles];

}  // namespace

namespace cfdb {
void set_last_error(const std::string &msg);  // context.cu: the message cfd_last_error returns
}

namespace {
cfd_status noalloc_fail(cfd_status s, const std::string &m) {
  cfdb::set_last_error(m);
  return s;
}
}  // namespace

extern "C" cfd_status cfd_evaluate_net_flux_noalloc(const cfd_flux_arrays *a, const cfd_config *cfg, void *stream) {
  if (!a || !cfg) return noalloc_fail(CFD_ERR_BAD_ARG, "null argument");
  const int NP = a->n_physical, NT = a->n_total;
  if (NP <= 0 || NT < NP) return noalloc_fail(CFD_ERR_BAD_ARG, "bad sizes");
  if (NP > kMaxCells || cfdb::flux_block_count(NP) > kMaxBlocks)
    return noalloc_fail(CFD_ERR_BAD_ARG, "cfd_evaluate_net_flux_noalloc handles at most " + std::to_string(kMaxCells) +
                                             " physical cells; got " + std::to_string(NP));
  const int diss = cfg->dissipation_type;
  if (diss != CFD_DISS_ROE && diss != CFD_DISS_LLF && diss != CFD_DISS_MOVERS && diss != CFD_DISS_RICCA &&
      diss != CFD_DISS_MOVERS_NWSC)
    return noalloc_fail(CFD_ERR_BAD_ARG, "dissipation type must be LLF, MOVERS, ROE, RICCA or MOVERS_NWSC");
  if (diss != CFD_DISS_ROE && diss != CFD_DISS_LLF && cfg->is_second_order && cfg->reconstruct_primitive)
    return noalloc_fail(CFD_ERR_BAD_ARG, "RICCA_2O and MOVERS_NWSC_2O limit the conserved variables");
  if (cfg->dissipation_type == CFD_DISS_LLF && cfg->is_second_order)
    return noalloc_fail(CFD_ERR_BAD_ARG, "LLF is first order only");
  if (cfg->muscl != CFD_MUSCL_REFERENCE || cfg->precision != CFD_PREC_FP64 || cfg->limiter < 0 || cfg->limiter > 4)
    return noalloc_fail(CFD_ERR_BAD_ARG, "only the reference MUSCL stencil in FP64 is available without allocation");
  if (!a->n_faces || !a->neighbours || !a->nx || !a->ny || !a->dl || !a->area || !a->inv_area || !a->degenerate ||
      !a->prim || !a->U || !a->net_flux || !a->dt || !a->min_dt)
    return noalloc_fail(CFD_ERR_BAD_ARG, "missing array");
  if (cfg->is_second_order && (!a->second_neighbours || !a->d1 || !a->d2))
    return noalloc_fail(CFD_ERR_BAD_ARG, "second order needs the limiter stencil arrays");

  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return noalloc_fail(CFD_ERR_NO_DEVICE, cudaGetErrorString(e));
  // The device address of the scratch array in the calling thread's current context (the
  // host-side name g_noalloc_scratch is not a device address).  It is looked up on every call,
  // not cached: after a device reset, or in a driver-API context other than the primary one, the
  // array lives at another address, and the lookup costs little once the module is loaded.
  // Nothing is shared between threads on the host.
  double *scratch = nullptr;
  e = cudaGetSymbolAddress(reinterpret_cast<void **>(&scratch), g_noalloc_scratch);
  if (e != cudaSuccess || !scratch)
    return noalloc_fail(CFD_ERR_CUDA, std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  cfdb::DevMesh m{};
  m.NP = NP;
  m.NT = NT;
  m.NB = 0;
  m.nf = a->n_faces;
  m.nbr = a->neighbours;
  m.nx = a->nx;
  m.ny = a->ny;
  m.dl = a->dl;
  m.area = a->area;
  m.inv_area = a->inv_area;
  m.n2 = a->second_neighbours;
  m.d1l = a->d1;
  m.d2l = a->d2;
  m.degen = a->degenerate;
  cfdb::DevState st{};
  st.U = const_cast<double *>(a->U);
  st.prim = const_cast<double *>(a->prim);
  st.R = a->net_flux;
  st.dtc = a->dt;
  st.ctl = scratch;
  st.counter = reinterpret_cast<unsigned int *>(scratch + kCtlDoubles);
  st.status = reinterpret_cast<int *>(scratch + kCtlDoubles) + 2;
  st.partial = scratch + kCtlDoubles + kCounterDoubles;
  cfdb::FluxParams fp{};
  fp.dissipation = cfg->dissipation_type;
  fp.movers_single = cfg->movers_single_alpha ? 1 : 0;
  fp.movers_efix = cfg->movers_entropy_fix ? 1 : 0;
  fp.second_order = cfg->is_second_order;
  fp.limiter = cfg->limiter;
  fp.recon_prim = cfg->reconstruct_primitive;
  fp.consistent = 0;
  fp.muscl = 0;
  fp.lanes = 1;
  fp.precision = CFD_PREC_FP64;
  fp.cfl = cfg->cfl;
  fp.zeta = cfg->limiter_zeta;
  fp.zeta1 = cfg->limiter_zeta1;

  // The control block (its "done" flag) and the completion counter must start at zero; the
  // partial minima are written before they are read.
  e = cudaMemsetAsync(scratch, 0, sizeof(double) * (kCtlDoubles + kCounterDoubles), s);
  if (e != cudaSuccess) return noalloc_fail(CFD_ERR_CUDA, std::string("cudaMemsetAsync: ") + cudaGetErrorString(e));
  cfdb::launch_flux(s, m, st, fp, 0);
  e = cudaGetLastError();
  if (e != cudaSuccess) return noalloc_fail(CFD_ERR_CUDA, std::string("flux launch: ") + cudaGetErrorString(e));
  e = cudaMemcpyAsync(a->min_dt, scratch + cfdb::CTL_DTMIN, sizeof(double), cudaMemcpyDeviceToDevice, s);
  if (e != cudaSuccess) return noalloc_fail(CFD_ERR_CUDA, std::string("cudaMemcpyAsync: ") + cudaGetErrorString(e));
  return CFD_OK;
}
