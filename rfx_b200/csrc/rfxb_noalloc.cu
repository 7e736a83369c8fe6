// rfxb_forward_noalloc: the forward step for callers that cannot allocate
// device memory.
//
// Some host programs own every byte of device memory through their own
// allocator (a framework's caching pool, an XLA-style runtime that hands a
// library only the buffers it declared), and others cannot accept the
// device-wide synchronisation that cudaMalloc/cudaFree may imply in the middle
// of a timed loop.  They cannot create a plan, because a plan allocates its
// state.  This entry point runs the same fused step kernel with all of that
// internal state (padded double-buffered fields, update coefficients, CPML
// psi, spacing tables, descriptor and work list) carved out of one file-scope
// device array of fixed size, RFXB_NOALLOC_BYTES.  It calls no cudaMalloc,
// cudaFree or allocating library routine.
//
// Properties a caller must know:
//  * every GPU that loads the library holds the array until the process exits;
//  * the first call on a device sets that device up with it current: it looks
//    up the array's device address (cudaGetSymbolAddress) and raises the step
//    kernel's dynamic shared-memory limit; make that first call before any
//    stream capture.  The address is kept for the life of the process, so a
//    cudaDeviceReset of that device leaves it stale: no call may follow one;
//  * every call uploads small host tables (descriptor, work list, CPML
//    profile, sources, probes) from memory that only lives during the call,
//    so a call on a stream that is capturing is refused with RFXB_E_INVALID;
//  * all calls share the array and it keeps the last call's contents: each
//    call clears what must start at zero (fields' guards, the second field
//    buffer, psi), so calls are independent, but two calls whose work
//    overlaps on the GPU (different streams, or different host threads) race
//    on the array and corrupt each other;
//  * one call starts from the caller's fields with zero CPML psi and returns
//    the fields after n_steps steps; psi is not carried between calls;
//  * DFT planes and gradient regions are not supported here (use a plan).
#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cstring>
#include <mutex>

#include "../../include/rfxb200.h"
#include "rfxb_common.cuh"

namespace rfxb {
template <int TY, int MODE, bool EM>
__global__ void fwd_step_kernel(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int, int);
size_t fwd_step_smem_bytes(int mode);
__global__ void pack_kernel(float*, const float*, RfxbInst);
__global__ void unpack_kernel(float*, const float*, RfxbInst);
__global__ void coef_kernel(RfxbInst, float*, float*, float*, float*, const float*, const float*, const float*,
                            const unsigned char*, unsigned char*, float);
void set_last_error(const char* msg);   // the message rfxb_last_error() returns
}  // namespace rfxb

using namespace rfxb;

#define RFXB_NOALLOC_BYTES (64ull << 20)

// The scratch every call uses.  In host code this name is only a stand-in for
// the symbol; its device address comes from cudaGetSymbolAddress below.
static __device__ __align__(256) unsigned char g_rfxb_noalloc_scratch[RFXB_NOALLOC_BYTES];

namespace {

int noalloc_fail(int code, const char* msg) {
  set_last_error(msg);
  return code;
}

// Per-device set-up, done once with that device current: the device address
// of the scratch array, and the step kernel's dynamic shared-memory opt-in
// (its stages take close to the 48 KB default).  Host threads may race to the
// first call: the lock makes one of them do the set-up, the atomic publishes
// the address to the others.
unsigned char* scratch_address(int* rc) {
  constexpr int kMaxDev = 64;
  static std::atomic<unsigned char*> addr[kMaxDev];
  static std::mutex mu;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDev) {
    *rc = noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: no current CUDA device");
    return nullptr;
  }
  unsigned char* a = addr[dev].load(std::memory_order_acquire);
  if (!a) {
    std::lock_guard<std::mutex> lock(mu);
    a = addr[dev].load(std::memory_order_relaxed);
    if (!a) {
      const cudaError_t ea = cudaFuncSetAttribute(reinterpret_cast<const void*>(fwd_step_kernel<8, 0, false>),
                                                  cudaFuncAttributeMaxDynamicSharedMemorySize,
                                                  (int)fwd_step_smem_bytes(0));
      if (ea != cudaSuccess) {
        *rc = noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: raising the step kernel's shared-memory limit failed");
        return nullptr;
      }
      void* p = nullptr;
      const cudaError_t e = cudaGetSymbolAddress(&p, g_rfxb_noalloc_scratch);
      if (e != cudaSuccess || p == nullptr) {
        *rc = noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: cudaGetSymbolAddress of the scratch array failed");
        return nullptr;
      }
      a = static_cast<unsigned char*>(p);
      addr[dev].store(a, std::memory_order_release);
    }
  }
  *rc = 0;
  return a;
}

size_t align256(size_t v) { return (v + 255) / 256 * 256; }

}  // namespace

extern "C" int rfxb_forward_noalloc(const RfxbDesc* d, const float* eps_r_dev, const float* sigma_dev,
                                    float* const* fields_dev, const RfxbStepIO* io, int step0, int n_steps,
                                    void* stream) {
  constexpr int TY = 8;
  if (!d || !eps_r_dev || !sigma_dev || !fields_dev)
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: null descriptor, materials or fields");
  for (int c = 0; c < 6; ++c)
    if (!fields_dev[c]) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: null field pointer");
  if (d->nx < 2 || d->ny < 2 || d->nz < 2) return noalloc_fail(RFXB_E_SHAPE, "rfxb_forward_noalloc: grid too small");
  if (!(d->dt > 0.0)) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: dt must be positive");
  if (step0 < 0 || n_steps < 0) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: negative step range");
  if (d->n_dft > 0) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: DFT planes need a plan");
  if (d->n_flux > 0) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: flux monitors need a plan");
  if (d->ntff_host) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: an NTFF box needs a plan");
  if (d->grad_box[0] < d->grad_box[1])
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: gradient regions need a plan");
  if (!d->inv_xe_host || !d->inv_xh_host || !d->inv_ye_host || !d->inv_yh_host || !d->inv_ze_host ||
      !d->inv_zh_host)
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: inverse spacing tables are required");
  const int ncp = d->cpml_axes ? d->cpml_layers : 0;
  const int ncp4 = (ncp + 3) / 4 * 4;
  if (ncp < 0 || ncp > 64) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: cpml_layers must be 0..64");
  if (ncp > 0 && (!d->cpml_b_host || !d->cpml_c_host || !d->cpml_kappa_host))
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: CPML profiles are required");
  const int dims[3] = {d->nx, d->ny, d->nz};
  for (int a = 0; a < 3; ++a)
    if (ncp > 0 && ((d->cpml_axes >> a) & 1u) && dims[a] < 2 * ncp)
      return noalloc_fail(RFXB_E_SHAPE, "rfxb_forward_noalloc: CPML slabs of one axis overlap");
  if (d->n_src < 0 || d->n_probe < 0)
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: negative source or probe count");
  if (d->n_src > 0 && !d->src_cells_host)
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: null source cell table");
  if (d->n_probe > 0 && !d->probe_cells_host)
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: null probe cell table");
  for (int s = 0; s < d->n_src; ++s) {
    const int32_t* c = d->src_cells_host + 4 * s;
    if (c[0] < 0 || c[0] >= d->nx || c[1] < 0 || c[1] >= d->ny || c[2] < 0 || c[2] >= d->nz || c[3] < 0 || c[3] > 2)
      return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: source cell or component out of range");
  }
  for (int p = 0; p < d->n_probe; ++p) {
    const int32_t* c = d->probe_cells_host + 4 * p;
    if (c[0] < 0 || c[0] >= d->nx || c[1] < 0 || c[1] >= d->ny || c[2] < 0 || c[2] >= d->nz || (c[3] & 7) > 5 ||
        (c[3] & ~(7 | RFXB_PROBE_PRESOURCE)) != 0)
      return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: probe cell or component out of range");
  }
  if (d->n_src > 0 && (!io || !io->src_wave_dev))
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: sources need a source table");

  // --- layout of the internal state (same as a plan's) ---
  RfxbInst I;
  std::memset(&I, 0, sizeof(I));
  I.nx = d->nx; I.ny = d->ny; I.nz = d->nz;
  I.zs = ((d->nz + 1) + 31) / 32 * 32;
  I.ps = (long long)(d->ny + 2) * I.zs;
  I.off0 = 32 + I.ps + I.zs;
  const long long elems = (32 + (long long)(d->nx + 2) * I.ps + I.zs + 64 + 31) / 32 * 32;
  I.cs = elems;
  long long psi_elems[3] = {0, 0, 0};
  if (ncp > 0) {
    if (d->cpml_axes & 1u) psi_elems[0] = 4LL * ncp * d->ny * I.zs;
    if (d->cpml_axes & 2u) psi_elems[1] = 4LL * d->nx * ncp * I.zs;
    if (d->cpml_axes & 4u) psi_elems[2] = 4LL * d->nx * d->ny * ncp4;
  }
  const int ty_tiles = (d->ny + TY - 1) / TY, tz_tiles = (d->nz + 31) / 32;
  const long long tiles = (long long)ty_tiles * tz_tiles;
  int sms = 148, dev = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  int chunks = (int)std::max<long long>(1, (4LL * sms * 4 + tiles - 1) / tiles);
  chunks = std::max(1, std::min(chunks, std::max(1, d->nx / 8)));
  const int xlen = (d->nx + chunks - 1) / chunks;
  const long long n_work = tiles * ((d->nx + xlen - 1) / xlen);

  size_t off = 0;
  const size_t o_inst = off; off = align256(off + sizeof(RfxbInst));
  const size_t o_work = off; off = align256(off + sizeof(RfxbWork) * (size_t)n_work);
  size_t o_tab[6];
  const int tab_n[6] = {d->nx, d->nx, d->ny, d->ny, d->nz, d->nz};
  for (int t = 0; t < 6; ++t) { o_tab[t] = off; off = align256(off + sizeof(float) * (size_t)(tab_n[t] + 2)); }
  const size_t o_cpb = off; off = align256(off + sizeof(float) * 18 * (size_t)std::max(ncp, 1));
  const size_t o_src = off; off = align256(off + sizeof(int4) * (size_t)std::max(d->n_src, 1));
  const size_t o_prb = off; off = align256(off + sizeof(int4) * (size_t)std::max(d->n_probe, 1));
  const size_t o_coef = off; off = align256(off + sizeof(float) * 3 * (size_t)elems);
  const size_t o_f0 = off; off = align256(off + sizeof(float) * 6 * (size_t)elems);
  const size_t o_f1 = off; off = align256(off + sizeof(float) * 6 * (size_t)elems);
  size_t o_psi[2][2][3];
  for (int s = 0; s < 2; ++s)
    for (int h = 0; h < 2; ++h)
      for (int a = 0; a < 3; ++a) {
        o_psi[s][h][a] = off;
        off = align256(off + sizeof(float) * (size_t)std::max<long long>(psi_elems[a], 1));
      }
  if (off > RFXB_NOALLOC_BYTES)
    return noalloc_fail(RFXB_E_NOMEM, "rfxb_forward_noalloc: the grid's internal state exceeds the fixed "
                                      "64 MiB scratch of this entry point (roughly 0.8 M cells); use a plan");

  int rc = 0;
  unsigned char* base = scratch_address(&rc);
  if (!base) return rc;
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
  if (cudaStreamIsCapturing(st, &cap) != cudaSuccess || cap != cudaStreamCaptureStatusNone)
    return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: the stream is capturing (or its capture state is "
                                        "unknown); this entry point uploads host tables that live only during "
                                        "the call");

  // --- descriptor pointers into the scratch ---
  float* coef = reinterpret_cast<float*>(base + o_coef);
  float* f0 = reinterpret_cast<float*>(base + o_f0);
  float* f1 = reinterpret_cast<float*>(base + o_f1);
  for (int c = 0; c < 6; ++c) { I.F[0][c] = f0 + c * elems; I.F[1][c] = f1 + c * elems; }
  I.ca = coef; I.cb = coef + elems; I.ce = coef + 2 * elems; I.ch = nullptr;
  I.ch0 = (float)d->dt / (float)kMu0;
  const float** tabs[6] = {&I.xe, &I.xh, &I.ye, &I.yh, &I.ze, &I.zh};
  const float* htabs[6] = {d->inv_xe_host, d->inv_xh_host, d->inv_ye_host, d->inv_yh_host, d->inv_ze_host,
                           d->inv_zh_host};
  I.ncp = ncp;
  I.ncp4 = ncp4;
  I.cpml_axes = ncp > 0 ? (d->cpml_axes & 7u) : 0u;
  I.cpb = reinterpret_cast<const float*>(base + o_cpb);
  for (int s = 0; s < 2; ++s)
    for (int a = 0; a < 3; ++a) {
      I.psH[s][a] = reinterpret_cast<float*>(base + o_psi[s][0][a]);
      I.psE[s][a] = reinterpret_cast<float*>(base + o_psi[s][1][a]);
    }
  I.pec_axes = d->pec_axes & 7u;
  I.emask = nullptr;
  I.nsrc = d->n_src; I.src = reinterpret_cast<const int4*>(base + o_src); I.src_ld = d->n_src;
  I.srcw = io ? io->src_wave_dev : nullptr;
  I.nprb = d->n_probe; I.prb = reinterpret_cast<const int4*>(base + o_prb); I.prb_ld = d->n_probe;
  I.prb_out = io ? io->probe_out_dev : nullptr;
  I.hist = nullptr;
  I.status = nullptr;

  auto ok = [](cudaError_t e) { return e == cudaSuccess; };
  // tables with zero guards at -1 and n
  for (int t = 0; t < 6; ++t) {
    float* dst = reinterpret_cast<float*>(base + o_tab[t]);
    if (!ok(cudaMemsetAsync(dst, 0, sizeof(float) * (size_t)(tab_n[t] + 2), st)) ||
        !ok(cudaMemcpyAsync(dst + 1, htabs[t], sizeof(float) * (size_t)tab_n[t], cudaMemcpyHostToDevice, st)))
      return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: table upload failed");
    *tabs[t] = dst + 1;
  }
  if (ncp > 0) {
    float tb[6 * 3 * 64];
    for (int f = 0; f < 6; ++f)
      for (int s = 0; s < ncp; ++s) {
        tb[(f * 3 + 0) * ncp + s] = d->cpml_b_host[f * ncp + s];
        tb[(f * 3 + 1) * ncp + s] = d->cpml_c_host[f * ncp + s];
        tb[(f * 3 + 2) * ncp + s] = 1.0f / d->cpml_kappa_host[f * ncp + s] - 1.0f;
      }
    for (int f = 0; f < 6; ++f) {
      if (!(d->cpml_cell[f] > 0.0)) return noalloc_fail(RFXB_E_INVALID, "rfxb_forward_noalloc: bad CPML cell size");
      I.ib[f] = (float)(1.0 / d->cpml_cell[f]);
    }
    if (!ok(cudaMemcpyAsync(base + o_cpb, tb, sizeof(float) * 18 * ncp, cudaMemcpyHostToDevice, st)))
      return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: CPML table upload failed");
  }
  if (d->n_src > 0 &&
      !ok(cudaMemcpyAsync(base + o_src, d->src_cells_host, sizeof(int4) * d->n_src, cudaMemcpyHostToDevice, st)))
    return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: source upload failed");
  if (d->n_probe > 0 &&
      !ok(cudaMemcpyAsync(base + o_prb, d->probe_cells_host, sizeof(int4) * d->n_probe, cudaMemcpyHostToDevice, st)))
    return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: probe upload failed");
  // work list, written in pieces from a stack buffer
  {
    RfxbWork buf[256];
    int nb = 0;
    size_t written = 0;
    for (int xa = 0; xa < d->nx; xa += xlen)
      for (int y = 0; y < ty_tiles; ++y)
        for (int z = 0; z < tz_tiles; ++z) {
          buf[nb++] = RfxbWork{0, y * TY, z * 32, xa, std::min(d->nx, xa + xlen)};
          if (nb == 256) {
            if (!ok(cudaMemcpyAsync(base + o_work + written, buf, sizeof(buf), cudaMemcpyHostToDevice, st)))
              return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: work list upload failed");
            written += sizeof(buf);
            nb = 0;
          }
        }
    if (nb > 0 && !ok(cudaMemcpyAsync(base + o_work + written, buf, sizeof(RfxbWork) * nb, cudaMemcpyHostToDevice, st)))
      return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: work list upload failed");
  }
  if (!ok(cudaMemcpyAsync(base + o_inst, &I, sizeof(RfxbInst), cudaMemcpyHostToDevice, st)))
    return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: descriptor upload failed");
  // everything that must start at zero: both field buffers (guards included),
  // the coefficient guards, psi
  if (!ok(cudaMemsetAsync(base + o_coef, 0, sizeof(float) * 3 * (size_t)elems, st)) ||
      !ok(cudaMemsetAsync(base + o_f0, 0, sizeof(float) * 6 * (size_t)elems, st)) ||
      !ok(cudaMemsetAsync(base + o_f1, 0, sizeof(float) * 6 * (size_t)elems, st)))
    return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: clearing the scratch failed");
  for (int s = 0; s < 2; ++s)
    for (int h = 0; h < 2; ++h)
      for (int a = 0; a < 3; ++a)
        if (!ok(cudaMemsetAsync(base + o_psi[s][h][a], 0, sizeof(float) * (size_t)std::max<long long>(psi_elems[a], 1),
                                st)))
          return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: clearing psi failed");

  const long long cells = (long long)d->nx * d->ny * d->nz;
  const int blocks = (int)std::min<long long>((cells + 255) / 256, 65535LL * 8);
  coef_kernel<<<blocks, 256, 0, st>>>(I, coef, coef + elems, coef + 2 * elems, nullptr, eps_r_dev, sigma_dev, nullptr,
                                      nullptr, nullptr, (float)d->dt);
  for (int c = 0; c < 6; ++c) pack_kernel<<<blocks, 256, 0, st>>>(I.F[0][c], fields_dev[c], I);
  const RfxbInst* dI = reinterpret_cast<const RfxbInst*>(base + o_inst);
  const RfxbWork* dW = reinterpret_cast<const RfxbWork*>(base + o_work);
  int par = 0;
  for (int s = 0; s < n_steps; ++s) {
    fwd_step_kernel<TY, 0, false><<<(unsigned)n_work, dim3(32, TY), fwd_step_smem_bytes(0), st>>>(dI, dW, nullptr, step0 + s,
                                                                                           step_sel(par, par ^ 1, par));
    par ^= 1;
  }
  for (int c = 0; c < 6; ++c) unpack_kernel<<<blocks, 256, 0, st>>>(fields_dev[c], I.F[par][c], I);
  if (!ok(cudaGetLastError())) return noalloc_fail(RFXB_E_LAUNCH, "rfxb_forward_noalloc: kernel launch failed");
  return 0;
}
