// Host side of the C ABI declared in include/rfxb200.h: plan and batch
// objects, device allocation, descriptor upload, launch sequencing and the
// CUDA-graph replay of step chunks.
#include <cuda.h>
#include <memory>
#include <mutex>
#include <set>
#include <cudaTypedefs.h>
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <queue>
#include <utility>
#include <vector>

#include "../../include/rfxb200.h"
#include "rfxb_common.cuh"

namespace rfxb {
template <int TY, int MODE, bool EM>
__global__ void fwd_step_kernel(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int, int);
size_t fwd_step_smem_bytes(int mode);
__global__ void dft_kernel(const RfxbInst*, const RfxbDftPlane*, int, int, int);
__global__ void pack_kernel(float*, const float*, RfxbInst);
__global__ void unpack_kernel(float*, const float*, RfxbInst);
__global__ void coef_kernel(RfxbInst, float*, float*, float*, float*, const float*, const float*,
                            const float*, const unsigned char*, unsigned char*, float);
__global__ void adj_pass_a(const RfxbInst*, const AdjInst*, const RfxbWork*, int, int, int);
__global__ void adj_pass_b(const RfxbInst*, const AdjInst*, const RfxbWork*, int, int, int);
__global__ void adj_init_kernel(const RfxbInst*, const AdjInst*, int, int, int);
__global__ void dft_adj_kernel(const RfxbInst*, const AdjInst*, const RfxbDftPlane*, int, int, int);
__global__ void ntff_adj_kernel(const RfxbInst*, const AdjInst*, const RfxbNtffFace*, int, int, int);
__global__ void flux_adj_kernel(const RfxbInst*, const AdjInst*, const RfxbFluxPlane*, int, int, int);
__global__ void box_energy_kernel(RfxbInst, int, int, int, int, int, int, int, const double*, const double*,
                                  const double*, double*);
__global__ void box_flux_kernel(RfxbInst, int, int, int, int, int, int, int, double*);
__global__ void flux_kernel(const RfxbInst*, const RfxbFluxPlane*, int, int, int);
__global__ void ntff_kernel(const RfxbInst*, const RfxbNtffFace*, int, int, int);
template <int TY, int MODE>
__global__ void adj_step_kernel(const RfxbInst*, const AdjInst*, const RfxbWork*, const CUtensorMap*, int, int, int,
                                int);
template <int TY, bool EM>
__global__ void fwd_persist_kernel(const RfxbInst*, int, RfxbFwdQueues, const CUtensorMap*, int, int);
template <int TY>
__global__ void adj_persist_kernel(const RfxbInst*, const AdjInst*, int, RfxbAdjQueues, const CUtensorMap*, int, int,
                                   int);
size_t adj_step_smem_bytes(int mode, int zp);
template <int TY>
__global__ void fwd2_step_kernel(const RfxbInst*, const RfxbWork2*, const CUtensorMap*, int, int);
size_t fwd2_step_smem_bytes();
}  // namespace rfxb

using namespace rfxb;

namespace {

constexpr int kTY = 8;

thread_local std::string g_last_error;

int fail(int code, const std::string& msg) {
  g_last_error = msg;
  return code;
}

#define RFXB_CUDA(call)                                                                         \
  do {                                                                                          \
    cudaError_t _e = (call);                                                                    \
    if (_e != cudaSuccess)                                                                      \
      return fail(RFXB_E_LAUNCH, std::string(#call) + ": " + cudaGetErrorString(_e));          \
  } while (0)

}  // namespace

namespace rfxb {
void set_last_error(const char* msg) { g_last_error = msg; }
}  // namespace rfxb

namespace {

int sm_count() {
  static int n = -1;
  if (n < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) n = 148;
  }
  return n;
}

// Shared memory of one SM (228 KB on B200).
int smem_per_sm() {
  static int n = -1;
  if (n < 0) {
    int dev = 0;
    cudaGetDevice(&dev);
    if (cudaDeviceGetAttribute(&n, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev) != cudaSuccess) n = 233472;
  }
  return n;
}

}  // namespace

struct RfxbPlan {
  RfxbInst inst{};             // host copy of the device descriptor
  int nx = 0, ny = 0, nz = 0;
  double dt = 0.0;
  long long elems = 0;         // floats per padded per-cell array
  int par = 0;                 // parity of the field buffers holding the current state
  int ppar = 0;                // parity of the CPML psi buffers holding the current state (a
                               // two-step pass flips the fields once and the psi twice)
  float* mid = nullptr;        // intermediate field state of two-step passes (F[2]), allocated on first use
  std::vector<void*> allocs;
  // per-cell and table arrays
  float* ca = nullptr; float* cb = nullptr; float* ce = nullptr; float* ch = nullptr;
  unsigned char* emask = nullptr;
  bool has_mu = false;
  std::vector<int4> src, prb;
  std::vector<RfxbDftDesc> dft;
  std::vector<float2*> dft_cmp;
  std::vector<long long> dft_cells;
  std::vector<RfxbFluxDesc> flux;
  bool has_ntff = false;
  RfxbNtffDesc ntff{};
  long long psi_elems[3] = {0, 0, 0};
  // history
  float* hist = nullptr;
  long long hist_cap = 0;      // floats
  long long hcells = 0;
  // checkpoints
  std::vector<float*> ckpt;
  std::vector<int> ckpt_valid;
  // adjoint
  AdjInst adj{};
  bool adj_alloc = false;
  int adj_par = 0;    // parity of the adjoint psi buffers
  int adj_fpar = 0;   // parity of the adjoint field buffers
  // single-plan group state
  RfxbBatch* self_group = nullptr;
  // TMA descriptors (layout in rfxb_inst.h, RFXB_NMAPS)
  CUtensorMap tmaps[RFXB_NMAPS];
  bool psi_maps_ok = false;    // the CPML psi maps encoded (staged-psi kernel usable)
  bool adj_psi_maps_ok = false;  // the same for the adjoint psi
  int l2promo = 2;             // L2 promotion of this plan's TMA maps: 0 none, 1 64 B, 2 128 B, 3 256 B

  ~RfxbPlan() {
    for (void* p : allocs) cudaFree(p);
  }

  template <typename T>
  int alloc(T** p, size_t count) {
    void* q = nullptr;
    if (count == 0) count = 1;
    cudaError_t e = cudaMalloc(&q, count * sizeof(T));
    if (e != cudaSuccess) return fail(RFXB_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    allocs.push_back(q);
    *p = static_cast<T*>(q);
    return 0;
  }
  int64_t bytes = 0;
};

// A cached CUDA graph of a launch sequence: kind 0 forward steps
// [step0, step0+k), kind 1 reverse steps [step0-k, step0) of the adjoint.
struct GraphKey {
  int kind, step0, k, par0, fpar0, dft, ppar0 = 0;
  bool operator<(const GraphKey& o) const {
    return std::tie(kind, step0, k, par0, fpar0, dft, ppar0) <
           std::tie(o.kind, o.step0, o.k, o.par0, o.fpar0, o.dft, o.ppar0);
  }
};

struct RfxbBatch {
  std::vector<RfxbPlan*> plans;
  RfxbInst* d_inst = nullptr;
  AdjInst* d_adj = nullptr;
  RfxbWork* d_work = nullptr;     // every tile (reverse steps; forward steps when not split)
  int n_work = 0;
  // forward steps split between the CPML-free kernel (list 1) and the
  // staged-psi kernel (list 2), launched side by side on two streams
  bool fwd_split = false;
  bool fwd_split_avail = false;   // both forward lists exist (fwd_split may be chosen)
  int fwd_order = 0;              // split forward: 0 plain-tile launch first, 1 CPML-tile launch first
  RfxbWork* d_wf1 = nullptr;
  int n_wf1 = 0;
  RfxbWork* d_wf2 = nullptr;
  int n_wf2 = 0;
  // reverse steps split the same way (list 1 on the CPML-free variant 3)
  bool adj_split = false;
  RfxbWork* d_wa1 = nullptr;
  int n_wa1 = 0;
  RfxbWork* d_wa2 = nullptr;
  int n_wa2 = 0;
  cudaStream_t side_stream = nullptr;
  cudaEvent_t ev_fork = nullptr, ev_join = nullptr;
  // reverse variant 4 (CPML work that reaches no y slab) on a third stream
  bool adj_lite = false;
  bool adj_lite_avail = false;    // the variant-4 lists exist (adj_lite may be chosen)
  int adj_order = 0;              // permutation index of the reverse launches (rfxb200.h)
  RfxbWork* d_wa2y = nullptr;   // variant 2 list when variant 4 takes the rest
  int n_wa2y = 0;
  RfxbWork* d_wa4 = nullptr;
  int n_wa4 = 0;
  cudaStream_t side2 = nullptr;
  cudaEvent_t ev_join2 = nullptr;
  // two-step passes (fwd_depth 2): the two-step kernel's tiles, and the
  // one-step work of a pass -- the other CPML-free tiles (variant 1) and the
  // CPML tiles (variant 2) -- launched once per step of the pass through the
  // intermediate buffer F[2]
  int fwd_depth = 1;
  bool fwd_depth_avail = false;
  RfxbWork2* d_wd = nullptr;
  int n_wd = 0;
  RfxbWork* d_wd1 = nullptr;
  int n_wd1 = 0;
  RfxbWork* d_wd2 = nullptr;
  int n_wd2 = 0;
  RfxbDftPlane* d_dft = nullptr;
  RfxbDftPlane* d_dfta = nullptr;   // the same planes with the adjoint call's cotangents
  std::vector<RfxbDftPlane> dfta;
  bool has_dft_cot = false;
  RfxbFluxPlane* d_flux = nullptr;
  RfxbFluxPlane* d_fluxa = nullptr;   // the same monitors with the adjoint call's cotangents
  std::vector<RfxbFluxPlane> fluxa;
  bool has_flux_cot = false;
  std::vector<RfxbFluxPlane> flux;
  int flux_blocks = 0;
  RfxbNtffFace* d_ntff = nullptr;
  RfxbNtffFace* d_ntffa = nullptr;   // the same faces with the adjoint call's cotangents
  std::vector<RfxbNtffFace> ntffa;
  bool has_ntff_cot = false;
  std::vector<RfxbNtffFace> ntff;   // six faces per plan with a box
  std::vector<long long> ntff_off;  // float2 offset of each face in its plan's buffers
  int ntff_blocks = 0;
  CUtensorMap* d_maps = nullptr;   // RFXB_NMAPS per plan
  int* d_status = nullptr;         // device status word of the group's launches
  // persistent step launches (one launch per step over the split lists)
  int* d_qctr = nullptr;           // [8]: fetch counters of the forward (3) and reverse (4) queues
  int fwd_persist = 0;             // 0: off; k >= 1: on, k-1 CTAs per SM try the CPML-free list first
  int adj_persist = 0;             // 0: off; 1: on
  int fault_cta = -1;              // test-only fault injection of the persistent kernels
  int wait_limit = rfxb::kWaitLimit;
  int adj_persist_grid = 0;        // CTAs of the persistent reverse launch (resident at once)
  int fwd_mode = 0;                // forward step kernel variant (see rfxb_fwd.cu)
  int adj_mode = -1;               // reverse step kernel variant (see rfxb_adj_fused.cu), -1 not chosen yet
  int adj_zp = 4;                  // z-psi row capacity of the mode-2 reverse ring
  std::vector<RfxbDftPlane> dft;
  int dft_blocks = 0;
  std::vector<void*> allocs;
  cudaStream_t cap_stream = nullptr;
  // captured step sequences by key, with the call counter of their last use
  // (least recently used evicted first)
  std::map<GraphKey, cudaGraphExec_t> graphs;
  std::map<GraphKey, unsigned long long> graph_use;
  unsigned long long graph_clock = 0;
  ~RfxbBatch() {
    for (auto& kv : graphs) cudaGraphExecDestroy(kv.second);
    if (cap_stream) cudaStreamDestroy(cap_stream);
    if (side_stream) cudaStreamDestroy(side_stream);
    if (side2) cudaStreamDestroy(side2);
    if (ev_fork) cudaEventDestroy(ev_fork);
    if (ev_join) cudaEventDestroy(ev_join);
    if (ev_join2) cudaEventDestroy(ev_join2);
    for (void* p : allocs) cudaFree(p);
  }
};

namespace {

// Work list: (TY x 32) tiles of (y, z), each over an x range [xa, xb).
// The x split is chosen for the whole group so the CTA count fills whole
// waves of the resident capacity (tail waves idle most SMs) while keeping
// x ranges long enough that the one-plane prologue of each CTA stays cheap.
int pick_chunks(long long tiles, int min_nx, int resident) {
  int best = 1;
  double best_eff = -1.0;
  for (int c = 1; c <= 64; ++c) {
    if (c > 1 && min_nx / c < 8) break;
    const long long total = tiles * c;
    const long long waves = (total + resident - 1) / resident;
    const double fill = (double)total / (double)(waves * resident);
    const double xlen = (double)min_nx / c;
    const double eff = fill * xlen / (xlen + 1.5);
    if (eff > best_eff + 1e-9) { best_eff = eff; best = c; }
  }
  return best;
}

void make_work(const RfxbPlan& p, int inst_index, int chunks, std::vector<RfxbWork>& out) {
  const int ty_tiles = (p.ny + kTY - 1) / kTY;
  const int tz_tiles = (p.nz + 31) / 32;
  chunks = std::max(1, std::min(chunks, p.nx));
  const int xlen = (p.nx + chunks - 1) / chunks;
  for (int xa = 0; xa < p.nx; xa += xlen)
    for (int y = 0; y < ty_tiles; ++y)
      for (int z = 0; z < tz_tiles; ++z)
        out.push_back(RfxbWork{inst_index, y * kTY, z * 32, xa, std::min(p.nx, xa + xlen)});
}

// Cost-balanced work list.  A CTA's time is modelled as the sum over its
// planes of 1 (a plain Yee tile-plane) plus `slab` for every CPML slab the
// plane and tile lie in, plus `prologue` plane-costs for its start-up (the
// extra planes it stages and the H it recomputes at xa-1).  Each tile's x
// line is cut into pieces of about equal cost; the piece size is chosen, over
// one to four waves of the resident CTA capacity, by simulating the block
// scheduler's greedy dispatch of the pieces in decreasing cost order (the
// order the list is emitted in), so heavy CPML tiles and large instances of a
// batch no longer set the step time.
// A run of planes [xa, xb) of one tile with its modelled per-plane cost:
// c, plus cx on the planes of the x slabs (i < ncpx or i >= nx - ncpx).
struct WorkSeg {
  int inst, y0, z0, xa, xb, nx, ncpx;
  double c, cx;
};

void balance_segments(const std::vector<WorkSeg>& segs, int resident, double prologue, std::vector<RfxbWork>& out) {
  out.clear();
  if (segs.empty()) return;
  auto plane_cost = [](const WorkSeg& t, int i) {
    return t.c + ((i < t.ncpx || i >= t.nx - t.ncpx) ? t.cx : 0.0);
  };
  std::vector<double> total(segs.size());
  double W = 0.0;
  for (size_t q = 0; q < segs.size(); ++q) {
    double t = 0.0;
    for (int i = segs[q].xa; i < segs[q].xb; ++i) t += plane_cost(segs[q], i);
    total[q] = t;
    W += t;
  }
  struct Item { RfxbWork w; double cost; int piece; };
  auto cut = [&](double T, std::vector<Item>& items) {
    items.clear();
    for (size_t q = 0; q < segs.size(); ++q) {
      const WorkSeg& t = segs[q];
      const int len = t.xb - t.xa;
      const int mmax = std::max(1, len / 4);   // pieces of at least 4 planes
      const int m = std::max(1, std::min(mmax, (int)std::llround(total[q] / T)));
      int xa = t.xa;
      double acc = 0.0;
      for (int piece = 1; piece <= m; ++piece) {
        const double goal = total[q] * piece / m;
        int xb = xa;
        double c = 0.0;
        while (xb < t.xb && (piece == m || acc + c + 0.5 * plane_cost(t, xb) <= goal)) {
          c += plane_cost(t, xb);
          ++xb;
        }
        if (xb == xa) { c += plane_cost(t, xb); ++xb; }
        items.push_back(Item{RfxbWork{t.inst, t.y0, t.z0, xa, xb}, c + prologue * t.c, piece});
        acc += c;
        xa = xb;
        if (xa >= t.xb) break;
      }
    }
    // decreasing cost in 5% buckets; within a bucket x-piece major, so tiles
    // that neighbour in (y, z) run the same x range together and share halos
    // through L2
    double cmax = 0.0;
    for (const Item& it : items) cmax = std::max(cmax, it.cost);
    auto bucket = [&](const Item& it) { return (int)std::floor(20.0 * it.cost / cmax); };
    std::stable_sort(items.begin(), items.end(), [&](const Item& a, const Item& b) {
      const int ba = bucket(a), bb = bucket(b);
      if (ba != bb) return ba > bb;
      return a.piece < b.piece;
    });
  };
  auto makespan = [&](const std::vector<Item>& items) {
    std::priority_queue<double, std::vector<double>, std::greater<double>> slots;
    for (int r = 0; r < resident; ++r) slots.push(0.0);
    double end = 0.0;
    for (const Item& it : items) {
      const double t = slots.top() + it.cost;
      slots.pop();
      slots.push(t);
      end = std::max(end, t);
    }
    return end;
  };
  std::vector<Item> best, cur;
  double best_t = 1e300;
  for (int waves = 1; waves <= 4; ++waves) {
    cut(W / ((double)resident * waves), cur);
    const double t = makespan(cur);
    if (t < best_t * (1.0 - 0.02)) { best_t = t; best = cur; }   // more waves only for a clear gain
  }
  for (const Item& it : best) out.push_back(it.w);
}

// Whether a forward tile's cells (rows y0-1 .. y0+TY-1, columns z0-1 ..
// z0+31) reach a y or z CPML slab.
bool tile_reaches_yz(const RfxbPlan& p, int y0, int z0) {
  const int n = p.inst.ncp;
  const unsigned ax = n > 0 ? p.inst.cpml_axes : 0u;
  return ((ax & 2u) && (y0 - 1 < n || y0 + kTY - 1 >= p.ny - n)) ||
         ((ax & 4u) && (z0 - 1 < n || z0 + 31 >= p.nz - n));
}

// Segments of every tile's full x line (cost model of the staged kernels).
void all_segments(const std::vector<RfxbPlan*>& plans, double slab, std::vector<WorkSeg>& segs) {
  for (size_t q = 0; q < plans.size(); ++q) {
    const RfxbPlan& p = *plans[q];
    const int n = p.inst.ncp;
    const unsigned ax = n > 0 ? p.inst.cpml_axes : 0u;
    for (int y0 = 0; y0 < p.ny; y0 += kTY)
      for (int z0 = 0; z0 < p.nz; z0 += 32) {
        double c = 1.0;
        if ((ax & 2u) && (y0 - 1 < n || y0 + kTY - 1 >= p.ny - n)) c += slab;
        if ((ax & 4u) && (z0 - 1 < n || z0 + 31 >= p.nz - n)) c += slab;
        const int ncpx = (ax & 1u) ? n : 0;
        segs.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, ncpx, c, (ax & 1u) ? slab : 0.0});
      }
  }
}

// Split of the forward work between the CPML-free kernel (variant 1) and the
// staged-psi kernel (variant 2): a tile that reaches no y/z slab runs planes
// ncp+1 .. nx-ncp-1 (whose x-1 prologue plane is outside the x slab too) on
// variant 1, everything else on variant 2.
void split_segments(const std::vector<RfxbPlan*>& plans, double slab, std::vector<WorkSeg>& plain,
                    std::vector<WorkSeg>& cpml) {
  for (size_t q = 0; q < plans.size(); ++q) {
    const RfxbPlan& p = *plans[q];
    const int n = p.inst.ncp;
    const unsigned ax = n > 0 ? p.inst.cpml_axes : 0u;
    for (int y0 = 0; y0 < p.ny; y0 += kTY)
      for (int z0 = 0; z0 < p.nz; z0 += 32) {
        if (ax == 0u) {
          plain.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, 0, 1.0, 0.0});
          continue;
        }
        const int ncpx = (ax & 1u) ? n : 0;
        const double cx = (ax & 1u) ? slab : 0.0;
        if (tile_reaches_yz(p, y0, z0)) {
          double c = 1.0;
          if ((ax & 2u) && (y0 - 1 < n || y0 + kTY - 1 >= p.ny - n)) c += slab;
          if ((ax & 4u) && (z0 - 1 < n || z0 + 31 >= p.nz - n)) c += slab;
          cpml.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, ncpx, c, cx});
          continue;
        }
        const int lo = ncpx > 0 ? ncpx + 1 : 0, hi = ncpx > 0 ? p.nx - ncpx : p.nx;
        if (hi - lo < 4) {
          cpml.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, ncpx, 1.0, cx});
          continue;
        }
        plain.push_back(WorkSeg{(int)q, y0, z0, lo, hi, p.nx, 0, 1.0, 0.0});
        if (lo > 0) cpml.push_back(WorkSeg{(int)q, y0, z0, 0, lo, p.nx, ncpx, 1.0, cx});
        if (hi < p.nx) cpml.push_back(WorkSeg{(int)q, y0, z0, hi, p.nx, p.nx, ncpx, 1.0, cx});
      }
  }
}

// The reverse step's split: its CPML terms reach rows y0-1 .. y0+TY, columns
// z0-1 .. z0+32 and planes xa-1 .. xb, so the CPML-free range of a tile that
// reaches no y/z slab is ncp+1 .. nx-ncp-2.
void split_adj_segments(const std::vector<RfxbPlan*>& plans, double slab, std::vector<WorkSeg>& plain,
                        std::vector<WorkSeg>& cpml, std::vector<WorkSeg>* cpml_noy = nullptr) {
  for (size_t q = 0; q < plans.size(); ++q) {
    const RfxbPlan& p = *plans[q];
    const int n = p.inst.ncp;
    const unsigned ax = n > 0 ? p.inst.cpml_axes : 0u;
    for (int y0 = 0; y0 < p.ny; y0 += kTY)
      for (int z0 = 0; z0 < p.nz; z0 += 32) {
        if (ax == 0u) {
          plain.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, 0, 1.0, 0.0});
          continue;
        }
        const int ncpx = (ax & 1u) ? n : 0;
        const double cx = (ax & 1u) ? slab : 0.0;
        const bool yz = ((ax & 2u) && (y0 - 1 < n || y0 + kTY >= p.ny - n)) ||
                        ((ax & 4u) && (z0 - 1 < n || z0 + 32 >= p.nz - n));
        const bool ys = (ax & 2u) && (y0 - 1 < n || y0 + kTY >= p.ny - n);
        // CPML work whose tile reaches no y slab goes to cpml_noy when given
        std::vector<WorkSeg>& dst = (cpml_noy && !ys) ? *cpml_noy : cpml;
        if (yz) {
          double c = 1.0;
          if (ys) c += slab;
          if ((ax & 4u) && (z0 - 1 < n || z0 + 32 >= p.nz - n)) c += slab;
          dst.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, ncpx, c, cx});
          continue;
        }
        const int lo = ncpx > 0 ? ncpx + 1 : 0, hi = ncpx > 0 ? p.nx - ncpx - 1 : p.nx;
        if (hi - lo < 4) {
          dst.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, ncpx, 1.0, cx});
          continue;
        }
        plain.push_back(WorkSeg{(int)q, y0, z0, lo, hi, p.nx, 0, 1.0, 0.0});
        if (lo > 0) dst.push_back(WorkSeg{(int)q, y0, z0, 0, lo, p.nx, ncpx, 1.0, cx});
        if (hi < p.nx) dst.push_back(WorkSeg{(int)q, y0, z0, hi, p.nx, p.nx, ncpx, 1.0, cx});
      }
  }
}

// Two-step passes.  A tile column (y0, z0) of plan p runs on the two-step
// kernel when every cell its two steps compute -- rows y0-2 .. y0+TY,
// columns z0-2 .. z0+32 -- lies out of every CPML slab, and no source, probe
// or gradient-history cell lies within reach (rows y0-2 .. y0+TY+1, columns
// z0-2 .. z0+33); the plan must have uniform H coefficients (a PEC edge mask
// is applied by the kernel).  On an axis without CPML the cells may reach the
// grid faces: such a
// column is a face column (the kernel's guarded path: zero outside the grid,
// PEC faces on E); 0 = not a two-step column, 1 = interior, 2 = face column.
bool depth2_plan(const RfxbPlan& p) { return p.inst.ch == nullptr; }

int depth2_column(const RfxbPlan& p, int y0, int z0) {
  if (y0 < 0 || y0 >= p.ny || z0 < 0 || z0 >= p.nz) return 0;
  const int n = p.inst.ncp;
  const unsigned ax = n > 0 ? p.inst.cpml_axes : 0u;
  if ((ax & 2u) && (y0 - 2 < n || y0 + kTY > p.ny - n - 1)) return 0;
  if ((ax & 4u) && (z0 - 2 < n || z0 + 32 > p.nz - n - 1)) return 0;
  auto near = [&](int j, int k) { return j >= y0 - 2 && j <= y0 + kTY + 1 && k >= z0 - 2 && k <= z0 + 33; };
  for (const int4& c : p.src)
    if (near(c.y, c.z)) return 0;
  for (const int4& c : p.prb)
    if (near(c.y, c.z)) return 0;
  const int* hb = p.inst.hb;
  if (hb[0] < hb[1] && hb[2] <= y0 + kTY + 1 && hb[3] - 1 >= y0 - 2 && hb[4] <= z0 + 33 && hb[5] - 1 >= z0 - 2)
    return 0;
  // interior: the first step's E cells (rows y0-1 .. y0+TY) off the faces,
  // its H cells (rows y0-2 ..) inside the grid
  const bool yin = y0 - 1 >= 1 && y0 + kTY <= p.ny - 2;
  const bool zin = z0 - 1 >= 1 && z0 + 32 <= p.nz - 2;
  return (yin && zin) ? 1 : 2;
}

// The x range of a plan's two-step segments: all planes without x CPML (the
// items at the x faces take the guarded path), else the planes whose x-1 ..
// x+1 neighbours are off the x slabs.
void depth2_xrange(const RfxbPlan& p, int& dlo, int& dhi) {
  const int n = p.inst.ncp;
  const int ncpx = (n > 0 && (p.inst.cpml_axes & 1u)) ? n : 0;
  dlo = ncpx > 0 ? ncpx + 1 : 0;
  dhi = ncpx > 0 ? p.nx - ncpx - 1 : p.nx;
}

// Work of a two-step pass: two-step segments (d2), the other CPML-free work
// (plain, variant 1) and the CPML work (cpml, variant 2; the same split as
// split_segments).  Together they cover every cell of every plan once.
void split_depth2_segments(const std::vector<RfxbPlan*>& plans, double slab, std::vector<WorkSeg>& d2,
                           std::vector<WorkSeg>& plain, std::vector<WorkSeg>& cpml) {
  for (size_t q = 0; q < plans.size(); ++q) {
    const RfxbPlan& p = *plans[q];
    const int n = p.inst.ncp;
    const unsigned ax = n > 0 ? p.inst.cpml_axes : 0u;
    const int ncpx = (ax & 1u) ? n : 0;
    const double cx = (ax & 1u) ? slab : 0.0;
    int dlo, dhi;
    depth2_xrange(p, dlo, dhi);
    const bool plan_ok = depth2_plan(p);
    for (int y0 = 0; y0 < p.ny; y0 += kTY)
      for (int z0 = 0; z0 < p.nz; z0 += 32) {
        int lo = 0, hi = p.nx;
        if (ax != 0u) {
          if (tile_reaches_yz(p, y0, z0)) {
            double c = 1.0;
            if ((ax & 2u) && (y0 - 1 < n || y0 + kTY - 1 >= p.ny - n)) c += slab;
            if ((ax & 4u) && (z0 - 1 < n || z0 + 31 >= p.nz - n)) c += slab;
            cpml.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, ncpx, c, cx});
            continue;
          }
          lo = ncpx > 0 ? ncpx + 1 : 0;
          hi = ncpx > 0 ? p.nx - ncpx : p.nx;
          if (hi - lo < 4) {
            cpml.push_back(WorkSeg{(int)q, y0, z0, 0, p.nx, p.nx, ncpx, 1.0, cx});
            continue;
          }
          if (lo > 0) cpml.push_back(WorkSeg{(int)q, y0, z0, 0, lo, p.nx, ncpx, 1.0, cx});
          if (hi < p.nx) cpml.push_back(WorkSeg{(int)q, y0, z0, hi, p.nx, p.nx, ncpx, 1.0, cx});
        }
        const int a = std::max(lo, dlo), b = std::min(hi, dhi);
        if (plan_ok && b - a >= 8 && depth2_column(p, y0, z0) > 0) {
          if (a < 2 && b > p.nx - 2 && b - a >= 32) {
            // the x faces' end pieces apart, so the rest takes the interior path
            d2.push_back(WorkSeg{(int)q, y0, z0, a, a + 8, p.nx, 0, 1.0, 0.0});
            d2.push_back(WorkSeg{(int)q, y0, z0, a + 8, b - 8, p.nx, 0, 1.0, 0.0});
            d2.push_back(WorkSeg{(int)q, y0, z0, b - 8, b, p.nx, 0, 1.0, 0.0});
          } else {
            d2.push_back(WorkSeg{(int)q, y0, z0, a, b, p.nx, 0, 1.0, 0.0});
          }
          if (a > lo) plain.push_back(WorkSeg{(int)q, y0, z0, lo, a, p.nx, 0, 1.0, 0.0});
          if (b < hi) plain.push_back(WorkSeg{(int)q, y0, z0, b, hi, p.nx, 0, 1.0, 0.0});
        } else {
          plain.push_back(WorkSeg{(int)q, y0, z0, lo, hi, p.nx, 0, 1.0, 0.0});
        }
      }
  }
}

// Where a two-step item also stores its intermediate state (RfxbWork2::mid):
// at its first / last plane when one-step work continues beyond it in x, on
// every plane when one of the eight neighbouring columns runs one-step work
// (its halo reads this tile) or when a DFT plane, flux monitor or NTFF face
// of the plan passes through the item (the observers read every step's
// state).  RFXB_MID_EDGE marks items whose cells reach a grid face.
int depth2_mid_flags(const RfxbPlan& p, const RfxbWork& w) {
  int dlo, dhi;
  depth2_xrange(p, dlo, dhi);
  int mid = 0;
  if (w.xa == dlo && dlo > 0) mid |= RFXB_MID_LO;
  if (w.xb == dhi && dhi < p.nx) mid |= RFXB_MID_HI;
  for (int dy = -1; dy <= 1; ++dy)
    for (int dz = -1; dz <= 1; ++dz) {
      const int y = w.y0 + dy * kTY, z = w.z0 + dz * 32;
      const bool in_grid = y >= 0 && y < p.ny && z >= 0 && z < p.nz;
      if ((dy || dz) && in_grid && depth2_column(p, y, z) == 0) mid |= RFXB_MID_ALL;
    }
  if (depth2_column(p, w.y0, w.z0) == 2 || w.xa < 2 || w.xb > p.nx - 2) mid |= RFXB_MID_EDGE;
  auto through = [&](int axis, int index) {
    const int lo = axis == 0 ? w.xa : axis == 1 ? w.y0 : w.z0;
    const int hi = axis == 0 ? w.xb : axis == 1 ? w.y0 + kTY : w.z0 + 32;
    return index + 1 >= lo && index - 1 < hi;   // the plane or a neighbour plane
  };
  for (const RfxbDftDesc& d : p.dft)
    if (through(d.axis, d.index)) mid |= RFXB_MID_ALL;
  for (const RfxbFluxDesc& f : p.flux)
    if (through(f.axis, f.index)) mid |= RFXB_MID_ALL;
  if (p.has_ntff) {
    const RfxbNtffDesc& b = p.ntff;
    if (through(0, b.i_lo) || through(0, b.i_hi) || through(1, b.j_lo) || through(1, b.j_hi) ||
        through(2, b.k_lo) || through(2, b.k_hi))
      mid |= RFXB_MID_ALL;
  }
  return mid;
}

void make_balanced_work(const std::vector<RfxbPlan*>& plans, int resident, double slab, double prologue,
                        std::vector<RfxbWork>& out) {
  std::vector<WorkSeg> segs;
  all_segments(plans, slab, segs);
  balance_segments(segs, resident, prologue, out);
}

// RFXB_WORK=uniform selects the plain split (one x chunk count for the group).
// Modelled extra cost of a tile-plane per CPML slab it lies in, relative to
// a plain tile-plane (RFXB_SLAB_WEIGHT, default 0.4).
double slab_weight() {
  static double v = -1.0;
  if (v < 0.0) {
    const char* e = getenv("RFXB_SLAB_WEIGHT");
    v = e ? std::max(0.0, atof(e)) : 0.4;
  }
  return v;
}

// RFXB_FWD_SPLIT=0 runs all forward tiles of a staged-psi group on one kernel.
bool fwd_split_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_FWD_SPLIT");
    v = (e && std::string(e) == "0") ? 0 : 1;
  }
  return v == 1;
}

// RFXB_ADJ_LITE=0 keeps the reverse CPML work of tiles without a y slab on
// variant 2 instead of variant 4.
bool adj_lite_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_ADJ_LITE");
    v = (e && std::string(e) == "0") ? 0 : 1;
  }
  return v == 1;
}

// Work-list builder: 1 cost-balanced (default), 0 RFXB_WORK=uniform (one x
// chunk count for the group), 2 RFXB_WORK=stream (x pieces of at most
// RFXB_WORK_PLANES planes, default 24, listed piece-major and then in raster
// order of instance, y, z, so that tiles which share halo rows are dispatched
// together and stay within a few planes of each other: their halo reads then
// come from L2).
int work_mode() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_WORK");
    v = (e && std::string(e) == "uniform") ? 0 : (e && std::string(e) == "stream") ? 2 : 1;
  }
  return v;
}

int stream_planes() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_WORK_PLANES");
    v = e ? std::max(4, atoi(e)) : 24;
  }
  return v;
}

void make_stream_work(const std::vector<RfxbPlan*>& plans, int planes, std::vector<RfxbWork>& out) {
  out.clear();
  std::vector<int> pieces(plans.size());
  int max_m = 0;
  for (size_t q = 0; q < plans.size(); ++q) {
    pieces[q] = std::max(1, (plans[q]->nx + planes / 2) / planes);
    max_m = std::max(max_m, pieces[q]);
  }
  for (int m = 0; m < max_m; ++m)
    for (size_t q = 0; q < plans.size(); ++q) {
      const RfxbPlan& p = *plans[q];
      if (m >= pieces[q]) continue;
      const int xa = (int)((long long)p.nx * m / pieces[q]);
      const int xb = (int)((long long)p.nx * (m + 1) / pieces[q]);
      for (int y0 = 0; y0 < p.ny; y0 += kTY)
        for (int z0 = 0; z0 < p.nz; z0 += 32) out.push_back(RfxbWork{(int)q, y0, z0, xa, xb});
    }
}

// Raise a kernel's dynamic shared memory limit once per device (the
// attribute belongs to the kernel in each device's context).
void allow_smem(const void* kernel, size_t bytes) {
  static std::mutex mu;
  static std::set<std::pair<int, const void*>> done;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  if (done.insert({dev, kernel}).second)
    cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
}

// Forward step kernel of a mode with its dynamic shared memory enabled.
using FwdKernel = void (*)(const RfxbInst*, const RfxbWork*, const CUtensorMap*, int, int);
FwdKernel fwd_kernel(int mode, bool em = false) {
  em = em && mode != 0;
  FwdKernel k = mode == 2 ? (em ? fwd_step_kernel<kTY, 2, true> : fwd_step_kernel<kTY, 2, false>)
                : mode == 1 ? (em ? fwd_step_kernel<kTY, 1, true> : fwd_step_kernel<kTY, 1, false>)
                            : fwd_step_kernel<kTY, 0, false>;
  allow_smem(reinterpret_cast<const void*>(k), fwd_step_smem_bytes(mode));
  return k;
}

// The two-step kernel with its dynamic shared memory enabled.
using Fwd2Kernel = void (*)(const RfxbInst*, const RfxbWork2*, const CUtensorMap*, int, int);
Fwd2Kernel fwd2_kernel() {
  Fwd2Kernel k = fwd2_step_kernel<kTY>;
  allow_smem(reinterpret_cast<const void*>(k), fwd2_step_smem_bytes());
  return k;
}

// CTAs of the two-step kernel resident at once.
int fwd2_resident() {
  static int r = -1;
  if (r < 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fwd2_kernel(), 32 * kTY, fwd2_step_smem_bytes()) !=
            cudaSuccess ||
        per_sm < 1)
      per_sm = 2;
    r = per_sm * sm_count();
  }
  return r;
}

// Default depth of the forward passes: RFXB_FWD_DEPTH=1 or 2 sets it for
// every group with two-step tiles; unset, groups without any CPML of at least
// 2^24 cells take two steps per pass (the 513^3 PEC benchmark: 78.1 -> 98.1
// G cells/s) and the others one (with CPML the gain measured 0-2 %, and on
// small grids the directly launched passes lose the graphs' launch rate;
// the autotuner chooses per workload).
int fwd_depth_default(const RfxbBatch* g) {
  const char* e = getenv("RFXB_FWD_DEPTH");
  if (e && std::string(e) == "2") return 2;
  if (e && std::string(e) == "1") return 1;
  long long cells = 0;
  for (const RfxbPlan* p : g->plans) {
    if (p->inst.ncp > 0 && p->inst.cpml_axes != 0u) return 1;
    cells += (long long)p->nx * p->ny * p->nz;
  }
  return cells >= (1LL << 24) ? 2 : 1;
}

using FwdPersistKernel = void (*)(const RfxbInst*, int, RfxbFwdQueues, const CUtensorMap*, int, int);
FwdPersistKernel fwd_persist_kernel_for(bool em) {
  FwdPersistKernel k = em ? fwd_persist_kernel<kTY, true> : fwd_persist_kernel<kTY, false>;
  allow_smem(reinterpret_cast<const void*>(k), fwd_step_smem_bytes(2));
  return k;
}

// CTAs of a persistent forward launch: as many as are resident at once.
int fwd_persist_grid(bool em) {
  static int r[2] = {-1, -1};
  if (r[em] < 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fwd_persist_kernel_for(em), 32 * kTY,
                                                      fwd_step_smem_bytes(2)) != cudaSuccess ||
        per_sm < 1)
      per_sm = 1;
    r[em] = per_sm * sm_count();
  }
  return r[em];
}

// Default of the persistent forward launch (RFXB_PERSIST=0 turns it off,
// =1 on with one plain-first CTA per SM; without the variable: off).
int fwd_persist_default() {
  const char* e = getenv("RFXB_PERSIST");
  if (!e) return 0;
  return std::string(e) == "0" ? 0 : 2;
}

// The persistent reverse launch needs the three reverse lists (variant 2 on
// y-slab tiles, variant 4 on the other CPML work, variant 3 on plain tiles).
bool adj_persist_avail(const RfxbBatch* g);

int resident_ctas(int mode) {
  static int r[3] = {-1, -1, -1};
  if (r[mode] < 0) {
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fwd_kernel(mode), 32 * kTY,
                                                      fwd_step_smem_bytes(mode)) != cudaSuccess ||
        per_sm < 1)
      per_sm = mode == 2 ? 3 : 4;
    r[mode] = per_sm * sm_count();
  }
  return r[mode];
}

// TMA staging is the default; RFXB_STAGING=cpasync selects per-thread 16-byte
// cp.async staging of the same planes.
bool use_tma() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_STAGING");
    v = (e && std::string(e) == "cpasync") ? 0 : 1;
  }
  return v == 1;
}

// L2 sector promotion of the TMA boxes.  The boxes' halo columns cover only
// part of a line, so promotion decides how much of the neighbour's line a
// halo miss drags in; which setting is fastest depends on the workload (the
// launch configuration's l2_promo field, chosen by the autotuner).  Default
// of a new plan: RFXB_L2PROMO = none | 64 | 128 | 256, else 128.
int l2_promotion_default() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_L2PROMO");
    const std::string m = e ? e : "128";
    v = m == "none" ? 0 : m == "64" ? 1 : m == "256" ? 3 : 2;
  }
  return v;
}

CUtensorMapL2promotion l2_promotion(int v) {
  return v == 0 ? CU_TENSOR_MAP_L2_PROMOTION_NONE
         : v == 1 ? CU_TENSOR_MAP_L2_PROMOTION_L2_64B
         : v == 3 ? CU_TENSOR_MAP_L2_PROMOTION_L2_256B
                  : CU_TENSOR_MAP_L2_PROMOTION_L2_128B;
}

// cuTensorMapEncodeTiled through the runtime's driver entry point, so the
// library needs no link-time dependency on libcuda.
PFN_cuTensorMapEncodeTiled_v12000 tensor_map_encoder() {
  static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
  static bool tried = false;
  if (!tried) {
    tried = true;
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(f);
  }
  return fn;
}

// 4-D map over a block of `ncomp` padded per-cell arrays with component stride
// cs: dims (zs, ny+2, nx+2, ncomp), origin at cell (i, j) = (-1, -1), k = 0.
int encode_block_map(CUtensorMap* m, const RfxbPlan& p, float* block, int ncomp, unsigned bx, unsigned by,
                     unsigned bc) {
  auto fn = tensor_map_encoder();
  if (!fn) return fail(RFXB_E_LAUNCH, "cuTensorMapEncodeTiled is not available from the driver");
  const RfxbInst& I = p.inst;
  void* addr = block + (I.off0 - I.ps - I.zs);
  cuuint64_t dims[4] = {(cuuint64_t)I.zs, (cuuint64_t)(p.ny + 2), (cuuint64_t)(p.nx + 2), (cuuint64_t)ncomp};
  cuuint64_t strides[3] = {(cuuint64_t)I.zs * 4, (cuuint64_t)I.ps * 4, (cuuint64_t)I.cs * 4};
  cuuint32_t box[4] = {bx, by, 1, bc};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, addr, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, l2_promotion(p.l2promo),
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(RFXB_E_LAUNCH, "cuTensorMapEncodeTiled failed (" + std::to_string((int)r) + ")");
  return 0;
}

// Map over the padded PEC edge-mask bytes: dims (zs, ny+2, nx+2, 1) with the
// origin at cell (-1, -1, 0), the tile box (32, TY, 1, 1).
int encode_emask_map(RfxbPlan* p) {
  auto fn = tensor_map_encoder();
  if (!fn) return fail(RFXB_E_LAUNCH, "cuTensorMapEncodeTiled is not available from the driver");
  const RfxbInst& I = p->inst;
  void* addr = p->emask + (I.off0 - I.ps - I.zs);
  cuuint64_t dims[4] = {(cuuint64_t)I.zs, (cuuint64_t)(p->ny + 2), (cuuint64_t)(p->nx + 2), 1};
  cuuint64_t strides[3] = {(cuuint64_t)I.zs, (cuuint64_t)I.ps, (cuuint64_t)I.ps * (cuuint64_t)(p->nx + 2)};
  cuuint32_t box[4] = {32, (cuuint32_t)kTY, 1, 1};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(&p->tmaps[RFXB_MAP_EMASK], CU_TENSOR_MAP_DATA_TYPE_UINT8, 4, addr, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, l2_promotion(p->l2promo),
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(RFXB_E_LAUNCH, "cuTensorMapEncodeTiled (edge mask) failed (" + std::to_string((int)r) + ")");
  return 0;
}

// 4-D map over one CPML psi array: dims (d0, d1, d2, 4 = side*2 + q), rows of
// d0 floats, box (b0, b1, 1, 2).
int encode_psi_map(CUtensorMap* m, float* base, long long d0, long long d1, long long d2, unsigned b0, unsigned b1,
                   int promo) {
  auto fn = tensor_map_encoder();
  if (!fn) return fail(RFXB_E_LAUNCH, "cuTensorMapEncodeTiled is not available from the driver");
  cuuint64_t dims[4] = {(cuuint64_t)d0, (cuuint64_t)d1, (cuuint64_t)d2, 4};
  cuuint64_t strides[3] = {(cuuint64_t)(d0 * 4), (cuuint64_t)(d0 * d1 * 4), (cuuint64_t)(d0 * d1 * d2 * 4)};
  cuuint32_t box[4] = {b0, b1, 1, 2};
  cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, base, dims, strides, box, estr,
                        CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, l2_promotion(promo),
                        CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  if (r != CUDA_SUCCESS) return fail(RFXB_E_LAUNCH, "cuTensorMapEncodeTiled (psi) failed (" + std::to_string((int)r) + ")");
  return 0;
}

int encode_psi_maps(RfxbPlan* p);

int encode_forward_maps(RfxbPlan* p) {
  const unsigned ty = kTY;
  for (int s = 0; s < 2; ++s) {
    if (int rc = encode_block_map(&p->tmaps[s], *p, p->inst.F[s][0], 6, 40, ty + 2, 3)) return rc;
    if (int rc = encode_block_map(&p->tmaps[2 + s], *p, p->inst.F[s][0], 6, 36, ty + 1, 3)) return rc;
  }
  if (int rc = encode_block_map(&p->tmaps[4], *p, p->ca, 3, 32, ty, 2)) return rc;
  if (int rc = encode_block_map(&p->tmaps[10], *p, p->ca, 3, 32, ty, 1)) return rc;
  // the two-step kernel's boxes (two-cell halo) and the intermediate state
  for (int s = 0; s < 2; ++s) {
    if (int rc = encode_block_map(&p->tmaps[RFXB_MAP_E2 + s], *p, p->inst.F[s][0], 6, 40, ty + 4, 3)) return rc;
    if (int rc = encode_block_map(&p->tmaps[RFXB_MAP_H2 + s], *p, p->inst.F[s][0], 6, 40, ty + 3, 3)) return rc;
  }
  if (int rc = encode_block_map(&p->tmaps[RFXB_MAP_C2], *p, p->ca, 3, 40, ty + 2, 2)) return rc;
  if (p->mid) {
    if (int rc = encode_block_map(&p->tmaps[RFXB_MAP_MIDE], *p, p->mid, 6, 40, ty + 2, 3)) return rc;
    if (int rc = encode_block_map(&p->tmaps[RFXB_MAP_MIDH], *p, p->mid, 6, 36, ty + 1, 3)) return rc;
  }
  const RfxbInst& I = p->inst;
  p->psi_maps_ok = false;
  if (I.ncp > 0) {
    // a psi map the driver refuses only rules out the staged-psi kernel
    const int rc = encode_psi_maps(p);
    p->psi_maps_ok = rc == 0;
  }
  return 0;
}

int encode_psi_maps(RfxbPlan* p) {
  const unsigned ty = kTY;
  const RfxbInst& I = p->inst;
  {
    const long long n = I.ncp, n4 = I.ncp4;
    for (int s = 0; s < 2; ++s) {
      if (I.cpml_axes & 1u) {
        if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_PSH + s], I.psH[s][0], I.zs, p->ny, n, 36, ty + 1, p->l2promo)) return rc;
        if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_PSE + s], I.psE[s][0], I.zs, p->ny, n, 32, ty, p->l2promo)) return rc;
      }
      if (I.cpml_axes & 2u) {
        if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_PSH + 2 + s], I.psH[s][1], I.zs, n, p->nx, 36, ty + 1, p->l2promo)) return rc;
        if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_PSE + 2 + s], I.psE[s][1], I.zs, n, p->nx, 32, ty, p->l2promo)) return rc;
      }
      if (I.cpml_axes & 4u) {
        if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_PSH + 4 + s], I.psH[s][2], n4, p->ny, p->nx, (unsigned)n4, ty + 1, p->l2promo))
          return rc;
        if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_PSE + 4 + s], I.psE[s][2], n4, p->ny, p->nx, (unsigned)n4, ty, p->l2promo))
          return rc;
      }
    }
  }
  return 0;
}

// Whether mode 2 (TMA-staged psi) can run a plan: the z-psi rows fit the
// ring, no tile reaches both slabs of an axis (its rows y0-1..y0+TY-1 or
// columns z0-1..z0+31), and psi offsets fit 32-bit arithmetic.
bool psi_staging_ok(const RfxbPlan& p) {
  const RfxbInst& I = p.inst;
  if (I.ncp == 0) return true;
  if (!p.psi_maps_ok || I.ncp4 > 16) return false;
  for (int a = 0; a < 3; ++a)
    if (p.psi_elems[a] >= (1LL << 31)) return false;
  const int n = I.ncp;
  if (I.cpml_axes & 2u)
    for (int y0 = 0; y0 < p.ny; y0 += kTY)
      if (y0 - 1 < n && y0 + kTY - 1 >= p.ny - n) return false;
  if (I.cpml_axes & 4u)
    for (int z0 = 0; z0 < p.nz; z0 += 32)
      if (z0 - 1 < n && z0 + 31 >= p.nz - n) return false;
  return true;
}

// Forward kernel variant of a group: 0 with RFXB_STAGING=cpasync or when a
// plan cannot stage its psi, 1 without any CPML, else 2.
// RFXB_FWD_MODE=2 runs CPML-free groups on the staged-psi variant too (a
// diagnostic of that variant's own cost).
int group_fwd_mode(const RfxbBatch* g) {
  if (!use_tma()) return 0;
  bool any_cpml = false;
  for (auto* p : g->plans) {
    if (p->inst.ncp > 0) any_cpml = true;
    if (!psi_staging_ok(*p)) return 0;
  }
  const char* e = getenv("RFXB_FWD_MODE");
  if (e && std::string(e) == "2") return 2;
  return any_cpml ? 2 : 1;
}

int encode_adjoint_maps(RfxbPlan* p) {
  const unsigned ty = kTY;
  for (int s = 0; s < 2; ++s) {
    if (int rc = encode_block_map(&p->tmaps[5 + s], *p, p->adj.aF[s][0], 6, 40, ty + 2, 3)) return rc;
    if (int rc = encode_block_map(&p->tmaps[7 + s], *p, p->adj.aF[s][0], 6, 36, ty + 1, 3)) return rc;
  }
  if (int rc = encode_block_map(&p->tmaps[9], *p, p->ca, 3, 40, ty + 2, 1)) return rc;
  if (int rc = encode_block_map(&p->tmaps[10], *p, p->ca, 3, 32, ty, 1)) return rc;
  if (int rc = encode_block_map(&p->tmaps[23], *p, p->ca, 3, 36, ty + 1, 1)) return rc;
  p->adj_psi_maps_ok = false;
  const RfxbInst& I = p->inst;
  if (I.ncp > 0) {
    // a psi map the driver refuses only rules out the staged-psi reverse kernel
    auto enc = [&]() -> int {
      const long long n = I.ncp, n4 = I.ncp4;
      for (int s = 0; s < 2; ++s) {
        if (I.cpml_axes & 1u) {
          if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_APE + s], p->adj.aPsiE[s][0], I.zs, p->ny, n, 36, ty + 1, p->l2promo))
            return rc;
          if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_APH + s], p->adj.aPsiH[s][0], I.zs, p->ny, n, 32, ty, p->l2promo))
            return rc;
        }
        if (I.cpml_axes & 2u) {
          if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_APE + 2 + s], p->adj.aPsiE[s][1], I.zs, n, p->nx, 40, ty + 2, p->l2promo))
            return rc;
          if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_APH + 2 + s], p->adj.aPsiH[s][1], I.zs, n, p->nx, 36, ty + 1, p->l2promo))
            return rc;
        }
        if (I.cpml_axes & 4u) {
          if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_APE + 4 + s], p->adj.aPsiE[s][2], n4, p->ny, p->nx,
                                      (unsigned)n4, ty + 2, p->l2promo))
            return rc;
          if (int rc = encode_psi_map(&p->tmaps[RFXB_MAP_APH + 4 + s], p->adj.aPsiH[s][2], n4, p->ny, p->nx,
                                      (unsigned)n4, ty + 1, p->l2promo))
            return rc;
        }
      }
      return 0;
    };
    p->adj_psi_maps_ok = enc() == 0;
  }
  return 0;
}

// Whether the staged-psi reverse kernel can run a plan: like the forward's
// test, over the cells its CPML terms touch (rows y0-1 .. y0+TY, columns
// z0-1 .. z0+32).
bool adj_psi_staging_ok(const RfxbPlan& p) {
  const RfxbInst& I = p.inst;
  if (I.ncp == 0) return true;
  if (!p.adj_psi_maps_ok || I.ncp4 > 16) return false;
  for (int a = 0; a < 3; ++a)
    if (p.psi_elems[a] >= (1LL << 31)) return false;
  const int n = I.ncp;
  if (I.cpml_axes & 2u)
    for (int y0 = 0; y0 < p.ny; y0 += kTY)
      if (y0 - 1 < n && y0 + kTY >= p.ny - n) return false;
  if (I.cpml_axes & 4u)
    for (int z0 = 0; z0 < p.nz; z0 += 32)
      if (z0 - 1 < n && z0 + 32 >= p.nz - n) return false;
  return true;
}

// Reverse kernel variant of a group: 0 with RFXB_STAGING=cpasync, 3 without
// any CPML, 2 when every plan can stage its psi, else 1; and the ring's
// z-row capacity.
void group_adj_mode(RfxbBatch* g) {
  g->adj_zp = 4;
  if (!use_tma()) { g->adj_mode = 0; return; }
  int mode = 2;
  bool any_cpml = false;
  for (auto* p : g->plans) {
    if (!adj_psi_staging_ok(*p)) mode = 1;
    if (p->inst.ncp > 0) any_cpml = true;
    g->adj_zp = std::max(g->adj_zp, p->inst.ncp4);
  }
  g->adj_mode = any_cpml ? mode : 3;   // no CPML anywhere: the lean variant
}

using AdjKernel = void (*)(const RfxbInst*, const AdjInst*, const RfxbWork*, const CUtensorMap*, int, int, int, int);
AdjKernel adj_kernel(int mode) {
  AdjKernel k = mode == 4   ? adj_step_kernel<kTY, 4>
                : mode == 3 ? adj_step_kernel<kTY, 3>
                : mode == 2 ? adj_step_kernel<kTY, 2>
                : mode == 1 ? adj_step_kernel<kTY, 1>
                            : adj_step_kernel<kTY, 0>;
  allow_smem(reinterpret_cast<const void*>(k), adj_step_smem_bytes(mode, 16));
  return k;
}

// Re-encode every TMA map a plan holds with its current L2 promotion (the
// maps are copied to the device before each launch sequence).
int reencode_maps(RfxbPlan* p) {
  if (int rc = encode_forward_maps(p)) return rc;
  if (p->emask)
    if (int rc = encode_emask_map(p)) return rc;
  if (p->adj_alloc)
    if (int rc = encode_adjoint_maps(p)) return rc;
  return 0;
}

int upload_tables(RfxbPlan* p, const float* h, int n, const float** dst) {
  std::vector<float> t(n + 2, 0.f);
  for (int i = 0; i < n; ++i) t[i + 1] = h[i];
  float* d = nullptr;
  if (int rc = p->alloc(&d, t.size())) return rc;
  RFXB_CUDA(cudaMemcpy(d, t.data(), t.size() * sizeof(float), cudaMemcpyHostToDevice));
  *dst = d + 1;
  return 0;
}

// The intermediate field buffer of two-step passes, allocated on first use
// with zero guards (no kernel writes a guard cell), and its tensor maps.
int ensure_mid(RfxbPlan* p) {
  if (p->mid) return 0;
  float* q = nullptr;
  if (int rc = p->alloc(&q, 6 * p->elems)) return rc;
  RFXB_CUDA(cudaMemset(q, 0, 6 * p->elems * sizeof(float)));
  p->mid = q;
  for (int c = 0; c < 6; ++c) p->inst.F[2][c] = q + c * p->elems;
  return encode_forward_maps(p);
}

int build_group(RfxbBatch* g) {
  std::vector<RfxbInst> insts;
  std::vector<RfxbWork> work;
  long long tiles = 0;
  int min_nx = 1 << 30;
  for (auto* p : g->plans) {
    tiles += (long long)((p->ny + kTY - 1) / kTY) * ((p->nz + 31) / 32);
    min_nx = std::min(min_nx, p->nx);
  }
  g->fwd_mode = group_fwd_mode(g);
  if (work_mode() == 1) {
    make_balanced_work(g->plans, resident_ctas(g->fwd_mode), g->fwd_mode == 2 ? slab_weight() : 1.0, 3.0, work);
  } else if (work_mode() == 2) {
    make_stream_work(g->plans, stream_planes(), work);
  } else {
    const int chunks = pick_chunks(tiles, min_nx, resident_ctas(g->fwd_mode));
    for (size_t q = 0; q < g->plans.size(); ++q) make_work(*g->plans[q], (int)q, chunks, work);
  }
  g->n_work = (int)work.size();
  auto galloc = [&](void** ptr, size_t bytes) -> int {
    cudaError_t e = cudaMalloc(ptr, std::max<size_t>(bytes, 16));
    if (e != cudaSuccess) return fail(RFXB_E_NOMEM, std::string("cudaMalloc: ") + cudaGetErrorString(e));
    g->allocs.push_back(*ptr);
    return 0;
  };
  // forward split (variant 2 groups, balanced lists; RFXB_FWD_SPLIT=0 starts
  // with the single list, which stays available as a launch configuration)
  g->fwd_split = false;
  if (g->fwd_mode == 2 && work_mode() == 1) {
    std::vector<WorkSeg> plain, cpml;
    split_segments(g->plans, slab_weight(), plain, cpml);
    std::vector<RfxbWork> w1, w2;
    balance_segments(plain, resident_ctas(1), 3.0, w1);
    balance_segments(cpml, resident_ctas(2), 3.0, w2);
    if (!w1.empty() && !w2.empty()) {
      if (int rc = galloc((void**)&g->d_wf1, sizeof(RfxbWork) * w1.size())) return rc;
      if (int rc = galloc((void**)&g->d_wf2, sizeof(RfxbWork) * w2.size())) return rc;
      RFXB_CUDA(cudaMemcpy(g->d_wf1, w1.data(), sizeof(RfxbWork) * w1.size(), cudaMemcpyHostToDevice));
      RFXB_CUDA(cudaMemcpy(g->d_wf2, w2.data(), sizeof(RfxbWork) * w2.size(), cudaMemcpyHostToDevice));
      g->n_wf1 = (int)w1.size();
      g->n_wf2 = (int)w2.size();
      RFXB_CUDA(cudaStreamCreateWithFlags(&g->side_stream, cudaStreamNonBlocking));
      RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming));
      RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming));
      g->fwd_split_avail = true;
      g->fwd_split = fwd_split_enabled();
    }
    // reverse split (used when the reverse kernel is variant 1 or 2); with
    // variant 2, the CPML work of tiles that reach no y slab can go to
    // variant 4 on a third stream
    std::vector<WorkSeg> aplain, acpml, aplain_b, ay, anoy;
    split_adj_segments(g->plans, slab_weight(), aplain, acpml);
    split_adj_segments(g->plans, slab_weight(), aplain_b, ay, &anoy);
    std::vector<RfxbWork> a1, a2;
    balance_segments(aplain, 4 * sm_count(), 3.0, a1);
    balance_segments(acpml, 3 * sm_count(), 3.0, a2);
    // (a grid with no CPML-free tile, e.g. one whose every z tile reaches a z
    // slab, still splits its CPML work between variants 2 and 4)
    if (!a2.empty()) {
      if (int rc = galloc((void**)&g->d_wa1, sizeof(RfxbWork) * std::max<size_t>(a1.size(), 1))) return rc;
      if (int rc = galloc((void**)&g->d_wa2, sizeof(RfxbWork) * a2.size())) return rc;
      if (!a1.empty())
        RFXB_CUDA(cudaMemcpy(g->d_wa1, a1.data(), sizeof(RfxbWork) * a1.size(), cudaMemcpyHostToDevice));
      RFXB_CUDA(cudaMemcpy(g->d_wa2, a2.data(), sizeof(RfxbWork) * a2.size(), cudaMemcpyHostToDevice));
      g->n_wa1 = (int)a1.size();
      g->n_wa2 = (int)a2.size();
      if (!g->side_stream) {
        RFXB_CUDA(cudaStreamCreateWithFlags(&g->side_stream, cudaStreamNonBlocking));
        RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming));
        RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming));
      }
      g->adj_split = true;
      std::vector<RfxbWork> a2y, a4;
      balance_segments(ay, 3 * sm_count(), 3.0, a2y);
      int zp = 4;
      for (auto* p : g->plans) zp = std::max(zp, p->inst.ncp4);
      // resident CTAs of variant 4: three per SM (its launch bounds give it
      // 80 registers)
      const int per_sm = 3;
      balance_segments(anoy, per_sm * sm_count(), 3.0, a4);
      if (!a4.empty()) {
        if (!a2y.empty()) {
          if (int rc = galloc((void**)&g->d_wa2y, sizeof(RfxbWork) * a2y.size())) return rc;
          RFXB_CUDA(cudaMemcpy(g->d_wa2y, a2y.data(), sizeof(RfxbWork) * a2y.size(), cudaMemcpyHostToDevice));
        }
        if (int rc = galloc((void**)&g->d_wa4, sizeof(RfxbWork) * a4.size())) return rc;
        RFXB_CUDA(cudaMemcpy(g->d_wa4, a4.data(), sizeof(RfxbWork) * a4.size(), cudaMemcpyHostToDevice));
        g->n_wa2y = (int)a2y.size();
        g->n_wa4 = (int)a4.size();
        RFXB_CUDA(cudaStreamCreateWithFlags(&g->side2, cudaStreamNonBlocking));
        RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_join2, cudaEventDisableTiming));
        g->adj_lite_avail = true;
        g->adj_lite = adj_lite_enabled();
      }
    }
  }
  // two-step pass lists (TMA groups on balanced lists): the two-step tiles
  // and the one-step work beside them; the pass itself is a launch
  // configuration (fwd_depth)
  g->fwd_depth_avail = false;
  g->fwd_depth = 1;
  if (g->fwd_mode >= 1 && work_mode() == 1) {
    std::vector<WorkSeg> d2, plain, cpml;
    split_depth2_segments(g->plans, slab_weight(), d2, plain, cpml);
    if (!d2.empty()) {
      std::vector<RfxbWork> wd, w1, w2;
      balance_segments(d2, fwd2_resident(), 3.0, wd);
      balance_segments(plain, resident_ctas(1), 3.0, w1);
      balance_segments(cpml, resident_ctas(2), 3.0, w2);
      std::vector<RfxbWork2> wd2;
      wd2.reserve(wd.size());
      for (const RfxbWork& w : wd)
        wd2.push_back(RfxbWork2{w.inst, w.y0, w.z0, w.xa, w.xb, depth2_mid_flags(*g->plans[w.inst], w)});
      if (int rc = galloc((void**)&g->d_wd, sizeof(RfxbWork2) * wd2.size())) return rc;
      RFXB_CUDA(cudaMemcpy(g->d_wd, wd2.data(), sizeof(RfxbWork2) * wd2.size(), cudaMemcpyHostToDevice));
      g->n_wd = (int)wd2.size();
      if (!w1.empty()) {
        if (int rc = galloc((void**)&g->d_wd1, sizeof(RfxbWork) * w1.size())) return rc;
        RFXB_CUDA(cudaMemcpy(g->d_wd1, w1.data(), sizeof(RfxbWork) * w1.size(), cudaMemcpyHostToDevice));
      }
      g->n_wd1 = (int)w1.size();
      if (!w2.empty()) {
        if (int rc = galloc((void**)&g->d_wd2, sizeof(RfxbWork) * w2.size())) return rc;
        RFXB_CUDA(cudaMemcpy(g->d_wd2, w2.data(), sizeof(RfxbWork) * w2.size(), cudaMemcpyHostToDevice));
      }
      g->n_wd2 = (int)w2.size();
      if (!g->side_stream) {
        RFXB_CUDA(cudaStreamCreateWithFlags(&g->side_stream, cudaStreamNonBlocking));
        RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_fork, cudaEventDisableTiming));
        RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_join, cudaEventDisableTiming));
      }
      if (!g->side2) {
        RFXB_CUDA(cudaStreamCreateWithFlags(&g->side2, cudaStreamNonBlocking));
        RFXB_CUDA(cudaEventCreateWithFlags(&g->ev_join2, cudaEventDisableTiming));
      }
      g->fwd_depth_avail = true;
      if (fwd_depth_default(g) == 2) {
        for (auto* p : g->plans)
          if (int rc = ensure_mid(p)) return rc;
        g->fwd_depth = 2;
      }
    }
  }
  if (int rc = galloc((void**)&g->d_inst, sizeof(RfxbInst) * g->plans.size())) return rc;
  if (int rc = galloc((void**)&g->d_adj, sizeof(AdjInst) * g->plans.size())) return rc;
  if (int rc = galloc((void**)&g->d_work, sizeof(RfxbWork) * work.size())) return rc;
  RFXB_CUDA(cudaMemcpy(g->d_work, work.data(), sizeof(RfxbWork) * work.size(), cudaMemcpyHostToDevice));
  // DFT planes
  g->dft.clear();
  int blocks = 0;
  for (size_t q = 0; q < g->plans.size(); ++q) {
    RfxbPlan* p = g->plans[q];
    for (size_t d = 0; d < p->dft.size(); ++d) {
      const RfxbDftDesc& dd = p->dft[d];
      RfxbDftPlane pl{};
      pl.inst = (int)q;
      pl.axis = dd.axis;
      pl.index = dd.index;
      pl.comp = dd.component;
      pl.nf = dd.n_freqs;
      pl.n1 = dd.axis == 0 ? p->ny : p->nx;
      pl.n2 = dd.axis == 2 ? p->ny : p->nz;
      pl.cmp = p->dft_cmp[d];
      pl.block0 = blocks;
      blocks += (int)((p->dft_cells[d] + 255) / 256);
      g->dft.push_back(pl);
    }
  }
  g->dft_blocks = blocks;
  // flux monitors (tangential components per normal axis, rfx/probes/probes.py:508-512)
  static const int kFluxComp[3][4] = {{RFXB_EY, RFXB_EZ, RFXB_HY, RFXB_HZ},
                                      {RFXB_EZ, RFXB_EX, RFXB_HZ, RFXB_HX},
                                      {RFXB_EX, RFXB_EY, RFXB_HX, RFXB_HY}};
  g->flux.clear();
  int fblocks = 0;
  for (size_t q = 0; q < g->plans.size(); ++q) {
    RfxbPlan* p = g->plans[q];
    for (const RfxbFluxDesc& fd : p->flux) {
      RfxbFluxPlane pl{};
      pl.inst = (int)q;
      pl.axis = fd.axis;
      pl.index = fd.index;
      pl.im1 = std::max(fd.index - 1, 0);
      pl.lo1 = fd.lo1;
      pl.n1 = fd.hi1 - fd.lo1;
      pl.lo2 = fd.lo2;
      pl.n2 = fd.hi2 - fd.lo2;
      pl.nf = fd.n_freqs;
      for (int t = 0; t < 4; ++t) pl.comp[t] = kFluxComp[fd.axis][t];
      pl.block0 = fblocks;
      fblocks += (pl.n1 * pl.n2 + 255) / 256;
      g->flux.push_back(pl);
    }
  }
  g->flux_blocks = fblocks;
  if (!g->flux.empty()) {
    if (int rc = galloc((void**)&g->d_flux, sizeof(RfxbFluxPlane) * g->flux.size())) return rc;
    if (int rc = galloc((void**)&g->d_fluxa, sizeof(RfxbFluxPlane) * g->flux.size())) return rc;
  }
  // NTFF boxes: faces x_lo, x_hi, y_lo, y_hi, z_lo, z_hi with the tangential
  // components of rfx/farfield.py:247-269
  static const int kNtffComp[3][4] = {{RFXB_EY, RFXB_EZ, RFXB_HY, RFXB_HZ},
                                      {RFXB_EX, RFXB_EZ, RFXB_HX, RFXB_HZ},
                                      {RFXB_EX, RFXB_EY, RFXB_HX, RFXB_HY}};
  g->ntff.clear();
  g->ntff_off.clear();
  int nblocks = 0;
  for (size_t q = 0; q < g->plans.size(); ++q) {
    RfxbPlan* p = g->plans[q];
    if (!p->has_ntff) continue;
    const RfxbNtffDesc& b = p->ntff;
    const int lo[3] = {b.i_lo, b.j_lo, b.k_lo}, hi[3] = {b.i_hi, b.j_hi, b.k_hi};
    long long off = 0;
    for (int f = 0; f < 6; ++f) {
      const int ax = f / 2, t1 = ax == 0 ? 1 : 0, t2 = ax == 2 ? 1 : 2;
      RfxbNtffFace A{};
      A.inst = (int)q;
      A.axis = ax;
      A.index = (f & 1) ? hi[ax] : lo[ax];
      A.lo1 = lo[t1];
      A.n1 = hi[t1] - lo[t1];
      A.lo2 = lo[t2];
      A.n2 = hi[t2] - lo[t2];
      A.nf = b.n_freqs;
      for (int t = 0; t < 4; ++t) A.comp[t] = kNtffComp[ax][t];
      A.block0 = nblocks;
      nblocks += (A.n1 * A.n2 + 255) / 256;
      g->ntff.push_back(A);
      g->ntff_off.push_back(off);
      off += (long long)A.nf * A.n1 * A.n2 * 4;
    }
  }
  g->ntff_blocks = nblocks;
  if (!g->ntff.empty()) {
    if (int rc = galloc((void**)&g->d_ntff, sizeof(RfxbNtffFace) * g->ntff.size())) return rc;
    if (int rc = galloc((void**)&g->d_ntffa, sizeof(RfxbNtffFace) * g->ntff.size())) return rc;
  }
  if (!g->dft.empty()) {
    if (int rc = galloc((void**)&g->d_dft, sizeof(RfxbDftPlane) * g->dft.size())) return rc;
    if (int rc = galloc((void**)&g->d_dfta, sizeof(RfxbDftPlane) * g->dft.size())) return rc;
  }
  if (int rc = galloc((void**)&g->d_maps, sizeof(CUtensorMap) * RFXB_NMAPS * g->plans.size())) return rc;
  if (int rc = galloc((void**)&g->d_status, sizeof(int))) return rc;
  RFXB_CUDA(cudaMemset(g->d_status, 0, sizeof(int)));
  if (int rc = galloc((void**)&g->d_qctr, 8 * sizeof(int))) return rc;
  RFXB_CUDA(cudaMemset(g->d_qctr, 0, 8 * sizeof(int)));
  g->fwd_persist = g->fwd_split_avail ? fwd_persist_default() : 0;
  g->adj_persist = (adj_persist_avail(g) && fwd_persist_default() > 0) ? 1 : 0;
  RFXB_CUDA(cudaStreamCreateWithFlags(&g->cap_stream, cudaStreamNonBlocking));
  return 0;
}

int upload_maps(RfxbBatch* g, cudaStream_t st) {
  std::vector<CUtensorMap> m(g->plans.size() * RFXB_NMAPS);
  for (size_t q = 0; q < g->plans.size(); ++q)
    std::memcpy(&m[q * RFXB_NMAPS], g->plans[q]->tmaps, sizeof(CUtensorMap) * RFXB_NMAPS);
  RFXB_CUDA(cudaMemcpyAsync(g->d_maps, m.data(), sizeof(CUtensorMap) * m.size(), cudaMemcpyHostToDevice, st));
  return 0;
}

// Upload descriptors with this call's IO pointers.
int upload_group(RfxbBatch* g, const RfxbStepIO* ios, bool* has_dft, bool* has_prb, bool* has_flux,
                 bool* has_ntff, cudaStream_t st) {
  std::vector<RfxbInst> insts(g->plans.size());
  *has_dft = false;
  *has_prb = false;
  size_t di = 0;
  for (size_t q = 0; q < g->plans.size(); ++q) {
    RfxbPlan* p = g->plans[q];
    insts[q] = p->inst;
    const RfxbStepIO* io = ios ? &ios[q] : nullptr;
    insts[q].srcw = io ? io->src_wave_dev : nullptr;
    if (p->inst.nsrc > 0 && insts[q].srcw == nullptr) insts[q].nsrc = 0;
    insts[q].prb_out = io ? io->probe_out_dev : nullptr;
    if (insts[q].prb_out) *has_prb = true;
    for (size_t d = 0; d < p->dft.size(); ++d, ++di) {
      const bool on = io && io->dft_acc_dev && io->dft_phase_dev && io->dft_acc_dev[d] && io->dft_phase_dev[d];
      g->dft[di].acc = on ? static_cast<float2*>(io->dft_acc_dev[d]) : nullptr;
      g->dft[di].phase = on ? static_cast<const float2*>(io->dft_phase_dev[d]) : nullptr;
      if (on) *has_dft = true;
    }
  }
  *has_flux = false;
  size_t fi = 0;
  for (size_t q = 0; q < g->plans.size(); ++q) {
    const RfxbStepIO* io = ios ? &ios[q] : nullptr;
    for (size_t d = 0; d < g->plans[q]->flux.size(); ++d, ++fi) {
      const bool on = io && io->flux_acc_dev && io->flux_kernel_dev && io->flux_acc_dev[d] && io->flux_kernel_dev[d];
      g->flux[fi].acc = on ? static_cast<double2*>(io->flux_acc_dev[d]) : nullptr;
      g->flux[fi].kern = on ? static_cast<const double2*>(io->flux_kernel_dev[d]) : nullptr;
      if (on) *has_flux = true;
    }
  }
  *has_ntff = false;
  for (size_t f = 0; f < g->ntff.size(); ++f) {
    RfxbNtffFace& A = g->ntff[f];
    const RfxbStepIO* io = ios ? &ios[A.inst] : nullptr;
    const bool on = io && io->ntff_acc_dev && io->ntff_cmp_dev && io->ntff_phase_dev;
    A.acc = on ? static_cast<float2*>(io->ntff_acc_dev) + g->ntff_off[f] : nullptr;
    A.cmp = on ? static_cast<float2*>(io->ntff_cmp_dev) + g->ntff_off[f] : nullptr;
    A.phase = on ? static_cast<const float2*>(io->ntff_phase_dev) : nullptr;
    if (on) *has_ntff = true;
  }
  for (const auto& A : g->ntff)
    if (*has_ntff && A.acc == nullptr)
      return fail(RFXB_E_INVALID, "either every NTFF box of a group gets accumulators and phase table, or none");
  if (!g->ntff.empty())
    RFXB_CUDA(cudaMemcpyAsync(g->d_ntff, g->ntff.data(), sizeof(RfxbNtffFace) * g->ntff.size(),
                              cudaMemcpyHostToDevice, st));
  for (const auto& pl : g->flux)
    if (*has_flux && pl.acc == nullptr)
      return fail(RFXB_E_INVALID, "either every flux monitor of a group gets accumulator and kernel, or none");
  if (!g->flux.empty())
    RFXB_CUDA(cudaMemcpyAsync(g->d_flux, g->flux.data(), sizeof(RfxbFluxPlane) * g->flux.size(),
                              cudaMemcpyHostToDevice, st));
  for (const auto& pl : g->dft)
    if (*has_dft && pl.acc == nullptr)
      return fail(RFXB_E_INVALID, "either every DFT plane of a group gets accumulator and phase table, or none");
  for (auto& I : insts) I.status = g->d_status;
  RFXB_CUDA(cudaMemcpyAsync(g->d_inst, insts.data(), sizeof(RfxbInst) * insts.size(), cudaMemcpyHostToDevice, st));
  if (int rc = upload_maps(g, st)) return rc;
  if (!g->dft.empty())
    RFXB_CUDA(cudaMemcpyAsync(g->d_dft, g->dft.data(), sizeof(RfxbDftPlane) * g->dft.size(),
                              cudaMemcpyHostToDevice, st));
  // cudaMemcpyAsync from pageable memory stages the source before returning
  return 0;
}

// Two-step passes run when chosen, when the group has two-step tiles and
// while every plan still has uniform H coefficients (materials set after the
// lists were built may add per-cell mu_r).
bool two_step(const RfxbBatch* g) {
  if (g->fwd_depth != 2 || !g->fwd_depth_avail) return false;
  for (const RfxbPlan* p : g->plans)
    if (!depth2_plan(*p)) return false;
  return true;
}

// Field and psi parities after n_steps steps from (par, ppar): a one-step
// launch flips both, a two-step pass flips the fields once and the psi twice.
void end_parities(const RfxbBatch* g, int n_steps, int& par, int& ppar) {
  for (int s = 0; s < n_steps;) {
    if (two_step(g) && s + 2 <= n_steps) { par ^= 1; s += 2; }
    else { par ^= 1; ppar ^= 1; ++s; }
  }
}

// One two-step pass over steps n, n+1 from fields F[par] and psi parity pp:
// the one-step work of step n (F[par] -> F[2], psi pp -> pp^1) runs beside
// the two-step tiles (F[par] -> F[par^1], intermediate state to F[2] where
// one-step work reads it), then the one-step work of step n+1
// (F[2] -> F[par^1], psi pp^1 -> pp).
int launch_pass(RfxbBatch* g, int n, int par, int pp, bool em, cudaStream_t st) {
  RFXB_CUDA(cudaEventRecord(g->ev_fork, st));
  RFXB_CUDA(cudaStreamWaitEvent(g->side_stream, g->ev_fork, 0));
  RFXB_CUDA(cudaStreamWaitEvent(g->side2, g->ev_fork, 0));
  fwd2_kernel()<<<g->n_wd, dim3(32, kTY), fwd2_step_smem_bytes(), g->side2>>>(g->d_inst, g->d_wd, g->d_maps, n, par);
  if (g->n_wd1 > 0)
    fwd_kernel(1, em)<<<g->n_wd1, dim3(32, kTY), fwd_step_smem_bytes(1), g->side_stream>>>(
        g->d_inst, g->d_wd1, g->d_maps, n, step_sel(par, 2, pp));
  if (g->n_wd2 > 0)
    fwd_kernel(2, em)<<<g->n_wd2, dim3(32, kTY), fwd_step_smem_bytes(2), st>>>(g->d_inst, g->d_wd2, g->d_maps, n,
                                                                            step_sel(par, 2, pp));
  RFXB_CUDA(cudaEventRecord(g->ev_join, g->side_stream));
  RFXB_CUDA(cudaEventRecord(g->ev_join2, g->side2));
  RFXB_CUDA(cudaStreamWaitEvent(st, g->ev_join, 0));
  RFXB_CUDA(cudaStreamWaitEvent(st, g->ev_join2, 0));
  if (g->n_wd1 > 0) {
    RFXB_CUDA(cudaEventRecord(g->ev_fork, st));
    RFXB_CUDA(cudaStreamWaitEvent(g->side_stream, g->ev_fork, 0));
    fwd_kernel(1, em)<<<g->n_wd1, dim3(32, kTY), fwd_step_smem_bytes(1), g->side_stream>>>(
        g->d_inst, g->d_wd1, g->d_maps, n + 1, step_sel(2, par ^ 1, pp ^ 1));
  }
  if (g->n_wd2 > 0)
    fwd_kernel(2, em)<<<g->n_wd2, dim3(32, kTY), fwd_step_smem_bytes(2), st>>>(g->d_inst, g->d_wd2, g->d_maps, n + 1,
                                                                            step_sel(2, par ^ 1, pp ^ 1));
  if (g->n_wd1 > 0) {
    RFXB_CUDA(cudaEventRecord(g->ev_join, g->side_stream));
    RFXB_CUDA(cudaStreamWaitEvent(st, g->ev_join, 0));
  }
  return 0;
}

int launch_steps(RfxbBatch* g, int step0, int n_steps, int par0, int ppar0, bool has_dft, bool has_flux,
                 bool has_ntff, cudaStream_t st) {
  int par = par0, pp = ppar0;
  bool em = false;   // stage the PEC edge masks when a plan of the group has one
  for (auto* p : g->plans) em = em || p->inst.emask != nullptr;
  // per-step observers of the state after step n, held in buffer b
  auto observe = [&](int n, int b) {
    if (has_dft) dft_kernel<<<g->dft_blocks, 256, 0, st>>>(g->d_inst, g->d_dft, (int)g->dft.size(), n, b);
    if (has_flux) flux_kernel<<<g->flux_blocks, 256, 0, st>>>(g->d_inst, g->d_flux, (int)g->flux.size(), n, b);
    if (has_ntff) ntff_kernel<<<g->ntff_blocks, 256, 0, st>>>(g->d_inst, g->d_ntff, (int)g->ntff.size(), n, b);
  };
  // the persistent launches clear their fetch counters when they finish;
  // clearing them here too keeps a sequence independent of earlier ones
  if (g->fwd_persist > 0 && g->fwd_split_avail) RFXB_CUDA(cudaMemsetAsync(g->d_qctr, 0, 4 * sizeof(int), st));
  for (int s = 0; s < n_steps;) {
    const int n = step0 + s;
    if (two_step(g) && s + 2 <= n_steps) {
      if (int rc = launch_pass(g, n, par, pp, em, st)) return rc;
      observe(n, 2);
      observe(n + 1, par ^ 1);
      par ^= 1;
      s += 2;
      continue;
    }
    const int sel = step_sel(par, par ^ 1, pp);
    if (g->fwd_persist > 0 && g->fwd_split_avail) {
      RfxbFwdQueues Q{};
      Q.list[0] = g->d_wf2;
      Q.count[0] = g->n_wf2;
      Q.list[1] = g->d_wf1;
      Q.count[1] = g->n_wf1;
      Q.ctr = g->d_qctr;
      Q.status = g->d_status;
      Q.plain_ctas = (g->fwd_persist - 1) * sm_count();
      Q.fault_cta = g->fault_cta;
      Q.wait_limit = g->wait_limit;
      fwd_persist_kernel_for(em)<<<fwd_persist_grid(em), dim3(32, kTY), fwd_step_smem_bytes(2), st>>>(
          g->d_inst, (int)g->plans.size(), Q, g->d_maps, n, sel);
    } else if (g->fwd_split) {
      // staged-psi tiles on the caller's stream, CPML-free tiles beside them
      RFXB_CUDA(cudaEventRecord(g->ev_fork, st));
      RFXB_CUDA(cudaStreamWaitEvent(g->side_stream, g->ev_fork, 0));
      // capture order (fwd_order): by default the plain tiles first
      // (measured 2 % faster on the sweep's forward phase than the CPML tiles
      // first, equal on one grid)
      auto plain = [&]() {
        fwd_kernel(1, em)<<<g->n_wf1, dim3(32, kTY), fwd_step_smem_bytes(1), g->side_stream>>>(g->d_inst, g->d_wf1,
                                                                                            g->d_maps, n, sel);
      };
      auto staged = [&]() {
        fwd_kernel(2, em)<<<g->n_wf2, dim3(32, kTY), fwd_step_smem_bytes(2), st>>>(g->d_inst, g->d_wf2, g->d_maps,
                                                                                n, sel);
      };
      if (g->fwd_order == 0) { plain(); staged(); }
      else { staged(); plain(); }
      RFXB_CUDA(cudaEventRecord(g->ev_join, g->side_stream));
      RFXB_CUDA(cudaStreamWaitEvent(st, g->ev_join, 0));
    } else {
      fwd_kernel(g->fwd_mode, em)<<<g->n_work, dim3(32, kTY), fwd_step_smem_bytes(g->fwd_mode), st>>>(
          g->d_inst, g->d_work, g->d_maps, n, sel);
    }
    observe(n, par ^ 1);
    par ^= 1;
    pp ^= 1;
    ++s;
  }
  RFXB_CUDA(cudaGetLastError());
  return 0;
}

// Launch sequences of more than a few steps are captured once into a CUDA
// graph (keyed by step range and parities) and replayed; the descriptors the
// kernels read are uploaded before each replay.  RFXB_GRAPHS=0 disables it.
bool graphs_enabled() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_GRAPHS");
    v = (e && std::string(e) == "0") ? 0 : 1;
  }
  return v == 1;
}

template <typename F>
int run_graph(RfxbBatch* g, const GraphKey& key, cudaStream_t st, F&& launch) {
  auto it = g->graphs.find(key);
  if (it == g->graphs.end()) {
    // Bound the cache.  A checkpointed run keeps one forward and one reverse
    // graph per segment alive (about 100 for 3000 steps at K = 64), so the
    // bound is well above that and the least recently used graph goes first.
    constexpr size_t kMaxGraphs = 512;
    cudaStreamCaptureStatus cap = cudaStreamCaptureStatusNone;
    cudaStreamIsCapturing(st, &cap);
    if (g->graphs.size() >= kMaxGraphs && cap == cudaStreamCaptureStatusNone) {
      auto victim = g->graphs.begin();
      unsigned long long oldest = ~0ull;
      for (auto v = g->graphs.begin(); v != g->graphs.end(); ++v) {
        const unsigned long long u = g->graph_use[v->first];
        if (u < oldest) { oldest = u; victim = v; }
      }
      // an executable graph destroyed while in flight is not cut short: the
      // runtime frees it when its launch completes, on whichever stream that
      // launch went, so no synchronisation is needed here
      cudaGraphExecDestroy(victim->second);
      g->graph_use.erase(victim->first);
      g->graphs.erase(victim);
    }
    RFXB_CUDA(cudaStreamBeginCapture(g->cap_stream, cudaStreamCaptureModeThreadLocal));
    const int rc = launch(g->cap_stream);
    cudaGraph_t graph = nullptr;
    const cudaError_t ec = cudaStreamEndCapture(g->cap_stream, &graph);
    if (rc) {
      if (graph) cudaGraphDestroy(graph);
      return rc;
    }
    if (ec != cudaSuccess) return fail(RFXB_E_LAUNCH, std::string("graph capture: ") + cudaGetErrorString(ec));
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ei = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ei != cudaSuccess) return fail(RFXB_E_LAUNCH, std::string("graph instantiate: ") + cudaGetErrorString(ei));
    it = g->graphs.emplace(key, exec).first;
  }
  g->graph_use[key] = ++g->graph_clock;
  RFXB_CUDA(cudaGraphLaunch(it->second, st));
  return 0;
}

int group_advance(RfxbBatch* g, const RfxbStepIO* ios, int step0, int n_steps, cudaStream_t st) {
  if (n_steps < 0 || step0 < 0) return fail(RFXB_E_INVALID, "negative step range");
  if (n_steps == 0) return 0;
  const int par0 = g->plans[0]->par, ppar0 = g->plans[0]->ppar;
  for (auto* p : g->plans)
    if (p->par != par0 || p->ppar != ppar0) return fail(RFXB_E_STATE, "plans of a batch must share the step parity");
  bool has_dft = false, has_prb = false, has_flux = false, has_ntff = false;
  if (int rc = upload_group(g, ios, &has_dft, &has_prb, &has_flux, &has_ntff, st)) return rc;
  // two-step passes launch directly: each pass is milliseconds of device
  // work, and their captured graphs measured slower to build and to replay
  // (1000 steps of a 513^3 grid: 0.9 s to capture, 1.58 s against 1.49 s per
  // replay)
  if (graphs_enabled() && n_steps >= 4 && !two_step(g)) {
    const GraphKey key{0, step0, n_steps, par0, 0, (has_dft ? 1 : 0) | (has_flux ? 2 : 0) | (has_ntff ? 4 : 0),
                       ppar0};
    if (int rc = run_graph(g, key, st, [&](cudaStream_t cs) {
          return launch_steps(g, step0, n_steps, par0, ppar0, has_dft, has_flux, has_ntff, cs);
        }))
      return rc;
  } else {
    if (int rc = launch_steps(g, step0, n_steps, par0, ppar0, has_dft, has_flux, has_ntff, st)) return rc;
  }
  int par = par0, ppar = ppar0;
  end_parities(g, n_steps, par, ppar);
  for (auto* p : g->plans) {
    p->par = par;
    p->ppar = ppar;
  }
  return 0;
}

bool adj_persist_avail(const RfxbBatch* g) { return g->adj_lite_avail && g->n_wa4 > 0 && g->n_wa1 > 0; }

using AdjPersistKernel = void (*)(const RfxbInst*, const AdjInst*, int, RfxbAdjQueues, const CUtensorMap*, int, int,
                                  int);
AdjPersistKernel adj_persist_kernel_for(int zp) {
  AdjPersistKernel k = adj_persist_kernel<kTY>;
  allow_smem(reinterpret_cast<const void*>(k), adj_step_smem_bytes(5, 16));
  (void)zp;
  return k;
}

int ensure_adjoint(RfxbPlan* p, cudaStream_t st) {
  if (!p->adj_alloc) {
    for (int s = 0; s < 2; ++s) {
      float* q = nullptr;
      if (int rc = p->alloc(&q, 6 * p->elems)) return rc;
      for (int c = 0; c < 6; ++c) p->adj.aF[s][c] = q + c * p->elems;
    }
    for (int s = 0; s < 2; ++s)
      for (int a = 0; a < 3; ++a) {
        if (int rc = p->alloc(&p->adj.aPsiH[s][a], p->psi_elems[a])) return rc;
        if (int rc = p->alloc(&p->adj.aPsiE[s][a], p->psi_elems[a])) return rc;
      }
    p->adj_alloc = true;
    if (int rc = encode_adjoint_maps(p)) return rc;
  }
  for (int s = 0; s < 2; ++s) RFXB_CUDA(cudaMemsetAsync(p->adj.aF[s][0], 0, 6 * p->elems * sizeof(float), st));
  for (int s = 0; s < 2; ++s)
    for (int a = 0; a < 3; ++a) {
      RFXB_CUDA(cudaMemsetAsync(p->adj.aPsiH[s][a], 0, std::max<long long>(1, p->psi_elems[a]) * sizeof(float), st));
      RFXB_CUDA(cudaMemsetAsync(p->adj.aPsiE[s][a], 0, std::max<long long>(1, p->psi_elems[a]) * sizeof(float), st));
    }
  p->adj_par = 0;
  p->adj_fpar = 0;
  return 0;
}

// The fused reverse step is the default; RFXB_ADJOINT_KERNEL=twopass selects
// the two unfused passes (an independent cross-check of the same transpose).
bool use_twopass() {
  static int v = -1;
  if (v < 0) {
    const char* e = getenv("RFXB_ADJOINT_KERNEL");
    v = (e && std::string(e) == "twopass") ? 1 : 0;
  }
  return v == 1;
}

int upload_adjoint(RfxbBatch* g, const RfxbAdjointIO* aios, cudaStream_t st) {
  std::vector<RfxbInst> insts(g->plans.size());
  std::vector<AdjInst> adjs(g->plans.size());
  for (size_t q = 0; q < g->plans.size(); ++q) {
    RfxbPlan* p = g->plans[q];
    const RfxbAdjointIO& a = aios[q];
    insts[q] = p->inst;
    insts[q].prb_out = nullptr;
    insts[q].srcw = nullptr;
    insts[q].g = a.g_dev;
    insts[q].g_ld = p->inst.nprb;
    insts[q].grad = a.grad_dev;
    insts[q].dca = a.dca_dev;
    insts[q].dcb = a.dcb_dev;
    insts[q].src_adj = a.src_adj_dev;
    if (a.grad_dev && (a.dca_dev == nullptr || a.dcb_dev == nullptr || p->hcells == 0))
      return fail(RFXB_E_STATE, "gradient requested without a gradient region or coefficient derivatives");
    adjs[q] = p->adj;
  }
  // DFT-plane cotangents (planes of the group in plan order, as in build_group)
  g->dfta = g->dft;
  g->has_dft_cot = false;
  size_t di = 0;
  for (size_t q = 0; q < g->plans.size(); ++q) {
    const RfxbAdjointIO& a = aios[q];
    for (size_t d = 0; d < g->plans[q]->dft.size(); ++d, ++di) {
      const bool on = a.dft_cot_dev && a.dft_phase_dev && a.dft_cot_dev[d] && a.dft_phase_dev[d];
      g->dfta[di].acc = on ? const_cast<float2*>(static_cast<const float2*>(a.dft_cot_dev[d])) : nullptr;
      g->dfta[di].cmp = nullptr;
      g->dfta[di].phase = on ? static_cast<const float2*>(a.dft_phase_dev[d]) : nullptr;
      if (on) g->has_dft_cot = true;
    }
  }
  if (!g->dfta.empty())
    RFXB_CUDA(cudaMemcpyAsync(g->d_dfta, g->dfta.data(), sizeof(RfxbDftPlane) * g->dfta.size(),
                              cudaMemcpyHostToDevice, st));
  // flux-monitor cotangents (monitors of the group in plan order)
  g->fluxa = g->flux;
  g->has_flux_cot = false;
  size_t fi = 0;
  for (size_t q = 0; q < g->plans.size(); ++q) {
    const RfxbAdjointIO& a = aios[q];
    for (size_t d = 0; d < g->plans[q]->flux.size(); ++d, ++fi) {
      const bool on = a.flux_cot_dev && a.flux_kernel_dev && a.flux_cot_dev[d] && a.flux_kernel_dev[d];
      g->fluxa[fi].acc = on ? const_cast<double2*>(static_cast<const double2*>(a.flux_cot_dev[d])) : nullptr;
      g->fluxa[fi].kern = on ? static_cast<const double2*>(a.flux_kernel_dev[d]) : nullptr;
      if (on) g->has_flux_cot = true;
    }
  }
  if (!g->fluxa.empty())
    RFXB_CUDA(cudaMemcpyAsync(g->d_fluxa, g->fluxa.data(), sizeof(RfxbFluxPlane) * g->fluxa.size(),
                              cudaMemcpyHostToDevice, st));
  // NTFF cotangents (faces of each plan's box at the offsets of the forward)
  g->ntffa = g->ntff;
  g->has_ntff_cot = false;
  for (size_t f = 0; f < g->ntffa.size(); ++f) {
    RfxbNtffFace& F = g->ntffa[f];
    const RfxbAdjointIO& a = aios[F.inst];
    const bool on = a.ntff_cot_dev && a.ntff_phase_dev;
    F.acc = on ? const_cast<float2*>(static_cast<const float2*>(a.ntff_cot_dev)) + g->ntff_off[f] : nullptr;
    F.cmp = nullptr;
    F.phase = on ? static_cast<const float2*>(a.ntff_phase_dev) : nullptr;
    if (on) g->has_ntff_cot = true;
  }
  if (!g->ntffa.empty())
    RFXB_CUDA(cudaMemcpyAsync(g->d_ntffa, g->ntffa.data(), sizeof(RfxbNtffFace) * g->ntffa.size(),
                              cudaMemcpyHostToDevice, st));
  for (auto& I : insts) I.status = g->d_status;
  RFXB_CUDA(cudaMemcpyAsync(g->d_inst, insts.data(), sizeof(RfxbInst) * insts.size(), cudaMemcpyHostToDevice, st));
  RFXB_CUDA(cudaMemcpyAsync(g->d_adj, adjs.data(), sizeof(AdjInst) * adjs.size(), cudaMemcpyHostToDevice, st));
  if (int rc = upload_maps(g, st)) return rc;
  return 0;
}

int group_adjoint_begin(RfxbBatch* g, const RfxbAdjointIO* aios, int n_total, cudaStream_t st) {
  if (n_total < 1) return fail(RFXB_E_INVALID, "n_total must be >= 1");
  for (auto* p : g->plans)
    if (int rc = ensure_adjoint(p, st)) return rc;
  if (int rc = upload_adjoint(g, aios, st)) return rc;
  adj_init_kernel<<<(unsigned)g->plans.size(), 32, 0, st>>>(g->d_inst, g->d_adj, (int)g->plans.size(), n_total - 1,
                                                             g->plans[0]->adj_fpar);
  if (g->has_dft_cot)   // DFT-plane cotangent of the last sample
    dft_adj_kernel<<<g->dft_blocks, 256, 0, st>>>(g->d_inst, g->d_adj, g->d_dfta, (int)g->dfta.size(), n_total - 1,
                                                  g->plans[0]->adj_fpar);
  if (g->has_ntff_cot)  // NTFF cotangent of the last sample
    ntff_adj_kernel<<<g->ntff_blocks, 256, 0, st>>>(g->d_inst, g->d_adj, g->d_ntffa, (int)g->ntffa.size(),
                                                    n_total - 1, g->plans[0]->adj_fpar);
  if (g->has_flux_cot)  // flux-monitor cotangent of the last sample
    flux_adj_kernel<<<g->flux_blocks, 256, 0, st>>>(g->d_inst, g->d_adj, g->d_fluxa, (int)g->fluxa.size(),
                                                    n_total - 1, g->plans[0]->adj_fpar);
  RFXB_CUDA(cudaGetLastError());
  return 0;
}

int group_adjoint_advance(RfxbBatch* g, const RfxbAdjointIO* aios, int step_hi, int n_steps, cudaStream_t st) {
  if (n_steps <= 0) return 0;
  if (step_hi - n_steps < 0) return fail(RFXB_E_INVALID, "reverse range reaches below step 0");
  const int par0 = g->plans[0]->adj_par;
  const int fpar0 = g->plans[0]->adj_fpar;
  for (auto* p : g->plans) {
    if (!p->adj_alloc) return fail(RFXB_E_STATE, "adjoint_advance before adjoint_begin");
    if (p->adj_par != par0 || p->adj_fpar != fpar0)
      return fail(RFXB_E_STATE, "plans of a batch must share the adjoint parity");
  }
  if (int rc = upload_adjoint(g, aios, st)) return rc;
  const bool two = use_twopass();
  if (g->adj_mode < 0) group_adj_mode(g);
  const int amode = g->adj_mode, zp = g->adj_zp;
  AdjKernel akern = two ? nullptr : adj_kernel(amode);
  const size_t asmem = adj_step_smem_bytes(amode, zp);
  auto launch = [&](cudaStream_t cs) -> int {
    int par = par0, fpar = fpar0;
    if (g->adj_persist && amode == 2 && adj_persist_avail(g))
      RFXB_CUDA(cudaMemsetAsync(g->d_qctr + 4, 0, 4 * sizeof(int), cs));
    for (int s = step_hi - 1; s >= step_hi - n_steps; --s) {
      if (two) {
        adj_pass_a<<<g->n_work, dim3(32, kTY), 0, cs>>>(g->d_inst, g->d_adj, g->d_work, s, par, fpar);
        adj_pass_b<<<g->n_work, dim3(32, kTY), 0, cs>>>(g->d_inst, g->d_adj, g->d_work, s, par, fpar);
      } else {
        if (g->adj_persist && amode == 2 && adj_persist_avail(g)) {
          RfxbAdjQueues Q{};
          Q.list[0] = g->d_wa2y;
          Q.count[0] = g->n_wa2y;
          Q.list[1] = g->d_wa4;
          Q.count[1] = g->n_wa4;
          Q.list[2] = g->d_wa1;
          Q.count[2] = g->n_wa1;
          Q.ctr = g->d_qctr + 4;
          Q.status = g->d_status;
          Q.role_ctas = sm_count();
          Q.fault_cta = g->fault_cta;
          Q.wait_limit = g->wait_limit;
          Q.zp = zp;
          const size_t psmem = adj_step_smem_bytes(5, zp);
          AdjPersistKernel pk = adj_persist_kernel_for(zp);
          if (g->adj_persist_grid <= 0) {
            int per_sm = 0;
            if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, pk, 32 * kTY, psmem) != cudaSuccess || per_sm < 1)
              per_sm = 1;
            g->adj_persist_grid = per_sm * sm_count();
          }
          pk<<<g->adj_persist_grid, dim3(32, kTY), psmem, cs>>>(g->d_inst, g->d_adj, (int)g->plans.size(), Q,
                                                               g->d_maps, s, par, fpar);
        } else if (g->adj_split && amode != 0) {
          // CPML tiles on the caller's stream, plain tiles beside them, and
          // (variant 2 groups) the CPML work without a y slab on variant 4
          const bool lite = g->adj_lite && amode == 2;
          RFXB_CUDA(cudaEventRecord(g->ev_fork, cs));
          RFXB_CUDA(cudaStreamWaitEvent(g->side_stream, g->ev_fork, 0));
          auto v2 = [&]() {
            if (lite) {
              if (g->n_wa2y > 0)
                akern<<<g->n_wa2y, dim3(32, kTY), asmem, cs>>>(g->d_inst, g->d_adj, g->d_wa2y, g->d_maps, s, par,
                                                               fpar, zp);
            } else {
              akern<<<g->n_wa2, dim3(32, kTY), asmem, cs>>>(g->d_inst, g->d_adj, g->d_wa2, g->d_maps, s, par, fpar,
                                                            zp);
            }
          };
          auto v4 = [&]() {
            if (lite)
              adj_kernel(4)<<<g->n_wa4, dim3(32, kTY), adj_step_smem_bytes(4, zp), g->side2>>>(
                  g->d_inst, g->d_adj, g->d_wa4, g->d_maps, s, par, fpar, zp);
          };
          auto v3 = [&]() {
            if (g->n_wa1 > 0)
              adj_kernel(3)<<<g->n_wa1, dim3(32, kTY), adj_step_smem_bytes(3, zp), g->side_stream>>>(
                  g->d_inst, g->d_adj, g->d_wa1, g->d_maps, s, par, fpar, zp);
          };
          // capture order = the order the graph hands the branches' CTAs to
          // the SMs (adj_order); the default 0 puts the largest, four-per-SM
          // variant 4 first, then the y-slab variant 2, the plain variant 3
          // last (measured best of the six orders, 3 % on the sweep's
          // reverse phase)
          if (lite) RFXB_CUDA(cudaStreamWaitEvent(g->side2, g->ev_fork, 0));
          static const char kOrder[6][3] = {{4, 2, 3}, {4, 3, 2}, {2, 4, 3}, {2, 3, 4}, {3, 4, 2}, {3, 2, 4}};
          for (int t = 0; t < 3; ++t) {
            const int v = kOrder[g->adj_order][t];
            if (v == 4) v4();
            else if (v == 2) v2();
            else v3();
          }
          RFXB_CUDA(cudaEventRecord(g->ev_join, g->side_stream));
          RFXB_CUDA(cudaStreamWaitEvent(cs, g->ev_join, 0));
          if (lite) {
            RFXB_CUDA(cudaEventRecord(g->ev_join2, g->side2));
            RFXB_CUDA(cudaStreamWaitEvent(cs, g->ev_join2, 0));
          }
        } else {
          akern<<<g->n_work, dim3(32, kTY), asmem, cs>>>(g->d_inst, g->d_adj, g->d_work, g->d_maps, s, par, fpar,
                                                         zp);
        }
        fpar ^= 1;
      }
      // DFT-plane cotangent of sample s-1 into the state the next reverse
      // step reads (the point where an E / H probe cotangent of s-1 lands)
      if (g->has_dft_cot && s >= 1)
        dft_adj_kernel<<<g->dft_blocks, 256, 0, cs>>>(g->d_inst, g->d_adj, g->d_dfta, (int)g->dfta.size(), s - 1,
                                                      fpar);
      if (g->has_ntff_cot && s >= 1)
        ntff_adj_kernel<<<g->ntff_blocks, 256, 0, cs>>>(g->d_inst, g->d_adj, g->d_ntffa, (int)g->ntffa.size(), s - 1,
                                                        fpar);
      if (g->has_flux_cot && s >= 1)
        flux_adj_kernel<<<g->flux_blocks, 256, 0, cs>>>(g->d_inst, g->d_adj, g->d_fluxa, (int)g->fluxa.size(), s - 1,
                                                        fpar);
      par ^= 1;
    }
    RFXB_CUDA(cudaGetLastError());
    return 0;
  };
  if (graphs_enabled() && n_steps >= 4) {
    const GraphKey key{1 + (two ? 1 : 0), step_hi, n_steps, par0, fpar0,
                       (g->has_dft_cot ? 1 : 0) | (g->has_ntff_cot ? 2 : 0) | (g->has_flux_cot ? 4 : 0)};
    if (int rc = run_graph(g, key, st, launch)) return rc;
  } else {
    if (int rc = launch(st)) return rc;
  }
  const int par = (par0 + n_steps) & 1;
  const int fpar = two ? fpar0 : ((fpar0 + n_steps) & 1);
  for (auto* p : g->plans) {
    p->adj_par = par;
    p->adj_fpar = fpar;
  }
  return 0;
}

}  // namespace

extern "C" {

int rfxb_version(void) { return 10000; }

const char* rfxb_last_error(void) { return g_last_error.c_str(); }

int rfxb_plan_create(const RfxbDesc* d, RfxbPlan** out) {
  if (!d || !out) return fail(RFXB_E_INVALID, "null descriptor or output");
  *out = nullptr;
  if (d->nx < 2 || d->ny < 2 || d->nz < 2) return fail(RFXB_E_SHAPE, "grid must be at least 2 cells on every axis");
  if ((long long)d->nx * d->ny * d->nz > (1LL << 34)) return fail(RFXB_E_SHAPE, "grid too large");
  if (!(d->dt > 0.0)) return fail(RFXB_E_INVALID, "dt must be positive");
  if (!d->inv_xe_host || !d->inv_xh_host || !d->inv_ye_host || !d->inv_yh_host || !d->inv_ze_host ||
      !d->inv_zh_host)
    return fail(RFXB_E_INVALID, "inverse spacing tables are required");
  const int ncp = d->cpml_layers;
  if (ncp < 0) return fail(RFXB_E_INVALID, "cpml_layers must be >= 0");
  if (ncp > 0) {
    if (!d->cpml_b_host || !d->cpml_c_host || !d->cpml_kappa_host)
      return fail(RFXB_E_INVALID, "CPML profiles are required when cpml_layers > 0");
    const int dims[3] = {d->nx, d->ny, d->nz};
    for (int a = 0; a < 3; ++a)
      if ((d->cpml_axes >> a) & 1u)
        if (dims[a] < 2 * ncp) return fail(RFXB_E_SHAPE, "CPML slabs of one axis overlap (axis shorter than 2*cpml_layers)");
  }
  if (d->n_src < 0 || d->n_probe < 0 || d->n_dft < 0 || d->n_flux < 0)
    return fail(RFXB_E_INVALID, "negative source, probe, DFT-plane or flux-monitor count");
  if ((d->n_src > 0 && !d->src_cells_host) || (d->n_probe > 0 && !d->probe_cells_host) ||
      (d->n_dft > 0 && !d->dft_host) || (d->n_flux > 0 && !d->flux_host))
    return fail(RFXB_E_INVALID, "null source, probe, DFT-plane or flux-monitor table with a positive count");
  for (int s = 0; s < d->n_src; ++s) {
    const int32_t* c = d->src_cells_host + 4 * s;
    if (c[0] < 0 || c[0] >= d->nx || c[1] < 0 || c[1] >= d->ny || c[2] < 0 || c[2] >= d->nz || c[3] < 0 || c[3] > 2)
      return fail(RFXB_E_INVALID, "source cell or component out of range");
  }
  for (int p = 0; p < d->n_probe; ++p) {
    const int32_t* c = d->probe_cells_host + 4 * p;
    if (c[0] < 0 || c[0] >= d->nx || c[1] < 0 || c[1] >= d->ny || c[2] < 0 || c[2] >= d->nz ||
        (c[3] & 7) > 5 || (c[3] & ~(7 | RFXB_PROBE_PRESOURCE)) != 0)
      return fail(RFXB_E_INVALID, "probe cell or component out of range");
  }
  for (int q = 0; q < d->n_dft; ++q) {
    const RfxbDftDesc& dd = d->dft_host[q];
    const int dims[3] = {d->nx, d->ny, d->nz};
    if (dd.axis < 0 || dd.axis > 2 || dd.index < 0 || dd.index >= dims[dd.axis] || dd.component < 0 ||
        dd.component > 5 || dd.n_freqs < 1)
      return fail(RFXB_E_INVALID, "DFT plane descriptor out of range");
  }
  for (int q = 0; q < d->n_flux; ++q) {
    const RfxbFluxDesc& fd = d->flux_host[q];
    const int dims[3] = {d->nx, d->ny, d->nz};
    if (fd.axis < 0 || fd.axis > 2 || fd.index < 0 || fd.index >= dims[fd.axis] || fd.n_freqs < 1)
      return fail(RFXB_E_INVALID, "flux monitor descriptor out of range");
    const int t1 = fd.axis == 0 ? d->ny : d->nx, t2 = fd.axis == 2 ? d->ny : d->nz;
    if (fd.lo1 < 0 || fd.hi1 > t1 || fd.lo1 >= fd.hi1 || fd.lo2 < 0 || fd.hi2 > t2 || fd.lo2 >= fd.hi2)
      return fail(RFXB_E_INVALID, "flux monitor region out of range or empty");
  }
  if (d->n_flux > 0 && !d->flux_host) return fail(RFXB_E_INVALID, "flux monitors need descriptors");
  if (const RfxbNtffDesc* b = d->ntff_host) {
    if (b->i_lo < 0 || b->i_lo >= b->i_hi || b->i_hi >= d->nx || b->j_lo < 0 || b->j_lo >= b->j_hi ||
        b->j_hi >= d->ny || b->k_lo < 0 || b->k_lo >= b->k_hi || b->k_hi >= d->nz || b->n_freqs < 1)
      return fail(RFXB_E_INVALID, "NTFF box out of range or empty");
  }
  const int* hb = d->grad_box;
  if (hb[0] < hb[1]) {
    if (hb[0] < 0 || hb[1] > d->nx || hb[2] < 0 || hb[3] > d->ny || hb[4] < 0 || hb[5] > d->nz || hb[2] >= hb[3] ||
        hb[4] >= hb[5])
      return fail(RFXB_E_INVALID, "gradient region out of range");
  }

  RfxbPlan* p = new RfxbPlan();
  p->nx = d->nx; p->ny = d->ny; p->nz = d->nz; p->dt = d->dt;
  RfxbInst& I = p->inst;
  I.nx = d->nx; I.ny = d->ny; I.nz = d->nz;
  I.zs = ((d->nz + 1) + 31) / 32 * 32;
  I.ps = (long long)(d->ny + 2) * I.zs;
  const long long base = 32;
  I.off0 = base + I.ps + I.zs;
  // a multiple of 32 elements, so every component block starts 128-byte aligned
  p->elems = (base + (long long)(d->nx + 2) * I.ps + I.zs + 64 + 31) / 32 * 32;
  I.cs = p->elems;
  auto bail = [&](int rc) { delete p; return rc; };
  for (int s = 0; s < 2; ++s) {
    float* q = nullptr;
    if (int rc = p->alloc(&q, 6 * p->elems)) return bail(rc);
    for (int c = 0; c < 6; ++c) I.F[s][c] = q + c * p->elems;
  }
  // ca, cb, ce in one block with the field component stride (one TMA map)
  if (int rc = p->alloc(&p->ca, 3 * p->elems)) return bail(rc);
  p->cb = p->ca + p->elems;
  p->ce = p->ca + 2 * p->elems;
  for (float* q : {p->ca, p->cb, p->ce})
    if (cudaMemset(q, 0, p->elems * sizeof(float)) != cudaSuccess) return bail(fail(RFXB_E_LAUNCH, "cudaMemset"));
  I.ca = p->ca; I.cb = p->cb; I.ce = p->ce; I.ch = nullptr;
  I.ch0 = (float)d->dt / (float)kMu0;
  if (int rc = upload_tables(p, d->inv_xe_host, d->nx, &I.xe)) return bail(rc);
  if (int rc = upload_tables(p, d->inv_xh_host, d->nx, &I.xh)) return bail(rc);
  if (int rc = upload_tables(p, d->inv_ye_host, d->ny, &I.ye)) return bail(rc);
  if (int rc = upload_tables(p, d->inv_yh_host, d->ny, &I.yh)) return bail(rc);
  if (int rc = upload_tables(p, d->inv_ze_host, d->nz, &I.ze)) return bail(rc);
  if (int rc = upload_tables(p, d->inv_zh_host, d->nz, &I.zh)) return bail(rc);
  // CPML
  I.ncp = ncp;
  I.cpml_axes = ncp > 0 ? (d->cpml_axes & 7u) : 0u;
  if (I.cpml_axes == 0) I.ncp = 0;
  I.ncp4 = (I.ncp + 3) / 4 * 4;
  if (I.ncp > 0) {
    std::vector<float> tb(6 * 3 * ncp);
    for (int f = 0; f < 6; ++f)
      for (int s = 0; s < ncp; ++s) {
        tb[(f * 3 + 0) * ncp + s] = d->cpml_b_host[f * ncp + s];
        tb[(f * 3 + 1) * ncp + s] = d->cpml_c_host[f * ncp + s];
        const float kap = d->cpml_kappa_host[f * ncp + s];
        tb[(f * 3 + 2) * ncp + s] = 1.0f / kap - 1.0f;  // rfx/boundaries/cpml.py:616
      }
    float* dcp = nullptr;
    if (int rc = p->alloc(&dcp, tb.size())) return bail(rc);
    if (cudaMemcpy(dcp, tb.data(), tb.size() * sizeof(float), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(RFXB_E_LAUNCH, "cudaMemcpy"));
    I.cpb = dcp;
    for (int f = 0; f < 6; ++f) {
      if (!(d->cpml_cell[f] > 0.0)) return bail(fail(RFXB_E_INVALID, "CPML cell sizes must be positive"));
      I.ib[f] = (float)(1.0 / d->cpml_cell[f]);
    }
    // (b, c / cell, (1/kappa - 1) / cell) per face and layer for the staged-psi kernel
    std::vector<float4> t4(6 * ncp);
    for (int f = 0; f < 6; ++f)
      for (int s = 0; s < ncp; ++s)
        t4[f * ncp + s] = make_float4(tb[(f * 3 + 0) * ncp + s], (float)((double)tb[(f * 3 + 1) * ncp + s] * I.ib[f]),
                                      (float)((double)tb[(f * 3 + 2) * ncp + s] * I.ib[f]), 0.f);
    float4* dct = nullptr;
    if (int rc = p->alloc(&dct, t4.size())) return bail(rc);
    if (cudaMemcpy(dct, t4.data(), t4.size() * sizeof(float4), cudaMemcpyHostToDevice) != cudaSuccess)
      return bail(fail(RFXB_E_LAUNCH, "cudaMemcpy"));
    I.cpt = dct;
    p->psi_elems[0] = 4LL * ncp * d->ny * I.zs;
    p->psi_elems[1] = 4LL * d->nx * ncp * I.zs;
    p->psi_elems[2] = 4LL * d->nx * d->ny * I.ncp4;
    for (int a = 0; a < 3; ++a) {
      if (!((I.cpml_axes >> a) & 1u)) { p->psi_elems[a] = 0; }
      for (int s = 0; s < 2; ++s) {
        float* q1 = nullptr; float* q2 = nullptr;
        if (int rc = p->alloc(&q1, p->psi_elems[a])) return bail(rc);
        if (int rc = p->alloc(&q2, p->psi_elems[a])) return bail(rc);
        I.psH[s][a] = q1;
        I.psE[s][a] = q2;
      }
    }
  }
  I.pec_axes = d->pec_axes & 7u;
  // sources / probes
  I.nsrc = d->n_src;
  I.nprb = d->n_probe;
  for (int s = 0; s < d->n_src; ++s) {
    const int32_t* c = d->src_cells_host + 4 * s;
    p->src.push_back(make_int4(c[0], c[1], c[2], c[3]));
  }
  for (int q = 0; q < d->n_probe; ++q) {
    const int32_t* c = d->probe_cells_host + 4 * q;
    p->prb.push_back(make_int4(c[0], c[1], c[2], c[3]));
  }
  int4* dsrc = nullptr; int4* dprb = nullptr;
  if (int rc = p->alloc(&dsrc, p->src.size())) return bail(rc);
  if (int rc = p->alloc(&dprb, p->prb.size())) return bail(rc);
  if (!p->src.empty() && cudaMemcpy(dsrc, p->src.data(), p->src.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(RFXB_E_LAUNCH, "cudaMemcpy"));
  if (!p->prb.empty() && cudaMemcpy(dprb, p->prb.data(), p->prb.size() * sizeof(int4), cudaMemcpyHostToDevice) != cudaSuccess)
    return bail(fail(RFXB_E_LAUNCH, "cudaMemcpy"));
  I.src = dsrc; I.src_ld = d->n_src;
  I.prb = dprb; I.prb_ld = d->n_probe;
  // DFT compensation buffers
  for (int q = 0; q < d->n_dft; ++q) {
    const RfxbDftDesc& dd = d->dft_host[q];
    p->dft.push_back(dd);
    const long long n1 = dd.axis == 0 ? d->ny : d->nx;
    const long long n2 = dd.axis == 2 ? d->ny : d->nz;
    float2* c = nullptr;
    if (int rc = p->alloc(&c, (size_t)dd.n_freqs * n1 * n2)) return bail(rc);
    p->dft_cmp.push_back(c);
    p->dft_cells.push_back(n1 * n2);
  }
  for (int q = 0; q < d->n_flux; ++q) p->flux.push_back(d->flux_host[q]);
  if (d->ntff_host) {
    p->has_ntff = true;
    p->ntff = *d->ntff_host;
  }
  for (int k = 0; k < 6; ++k) I.hb[k] = hb[k];
  if (hb[0] >= hb[1]) { I.hb[0] = 0; I.hb[1] = 0; }
  p->hcells = (long long)(I.hb[1] - I.hb[0]) * (I.hb[3] - I.hb[2]) * (I.hb[5] - I.hb[4]);
  I.hist = nullptr;
  std::memset(p->tmaps, 0, sizeof(p->tmaps));
  p->l2promo = l2_promotion_default();
  if (int rc = encode_forward_maps(p)) return bail(rc);
  // own single-plan group
  RfxbBatch* g = new RfxbBatch();
  g->plans.push_back(p);
  if (int rc = build_group(g)) { delete g; return bail(rc); }
  p->self_group = g;
  if (cudaDeviceSynchronize() != cudaSuccess) { delete g; return bail(fail(RFXB_E_LAUNCH, "setup failed")); }
  if (int rc = rfxb_plan_reset(p, nullptr)) { delete g; return bail(rc); }
  if (cudaStreamSynchronize(nullptr) != cudaSuccess) { delete g; return bail(fail(RFXB_E_LAUNCH, "reset failed")); }
  *out = p;
  return 0;
}

void rfxb_plan_destroy(RfxbPlan* p) {
  if (!p) return;
  cudaDeviceSynchronize();
  delete p->self_group;
  delete p;
}

int rfxb_plan_set_materials(RfxbPlan* p, const float* eps_r, const float* sigma, const float* mu_r,
                            const uint8_t* edge_mask, void* stream) {
  if (!p || !eps_r || !sigma) return fail(RFXB_E_INVALID, "plan, eps_r and sigma are required");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  if (mu_r && !p->ch) {
    if (int rc = p->alloc(&p->ch, p->elems)) return rc;
    RFXB_CUDA(cudaMemsetAsync(p->ch, 0, p->elems * sizeof(float), st));
  }
  p->inst.ch = mu_r ? p->ch : nullptr;
  if (edge_mask && !p->emask) {
    if (int rc = p->alloc(&p->emask, p->elems)) return rc;
    RFXB_CUDA(cudaMemsetAsync(p->emask, 0, p->elems, st));
    if (int rc = encode_emask_map(p)) return rc;
  }
  p->inst.emask = edge_mask ? p->emask : nullptr;
  const long long cells = (long long)p->nx * p->ny * p->nz;
  const int blocks = (int)std::min<long long>((cells + 255) / 256, 65535LL * 8);
  coef_kernel<<<blocks, 256, 0, st>>>(p->inst, p->ca, p->cb, p->ce, mu_r ? p->ch : nullptr, eps_r, sigma, mu_r,
                                      edge_mask, edge_mask ? p->emask : nullptr, (float)p->dt);
  RFXB_CUDA(cudaGetLastError());
  return 0;
}

int rfxb_plan_reset(RfxbPlan* p, void* stream) {
  if (!p) return fail(RFXB_E_INVALID, "null plan");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  for (int s = 0; s < 2; ++s)
    for (int c = 0; c < 6; ++c) RFXB_CUDA(cudaMemsetAsync(p->inst.F[s][c], 0, p->elems * sizeof(float), st));
  for (int s = 0; s < 2; ++s)
    for (int a = 0; a < 3; ++a) {
      if (p->psi_elems[a] > 0) {
        RFXB_CUDA(cudaMemsetAsync(p->inst.psH[s][a], 0, p->psi_elems[a] * sizeof(float), st));
        RFXB_CUDA(cudaMemsetAsync(p->inst.psE[s][a], 0, p->psi_elems[a] * sizeof(float), st));
      }
    }
  for (size_t q = 0; q < p->dft_cmp.size(); ++q)
    RFXB_CUDA(cudaMemsetAsync(p->dft_cmp[q], 0, p->dft[q].n_freqs * p->dft_cells[q] * sizeof(float2), st));
  p->par = 0;
  p->ppar = 0;
  return 0;
}

int rfxb_plan_load_fields(RfxbPlan* p, const float* const* fields, void* stream) {
  if (!p || !fields) return fail(RFXB_E_INVALID, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long cells = (long long)p->nx * p->ny * p->nz;
  const int blocks = (int)std::min<long long>((cells + 255) / 256, 65535LL * 8);
  for (int c = 0; c < 6; ++c) {
    if (!fields[c]) return fail(RFXB_E_INVALID, "null field pointer");
    pack_kernel<<<blocks, 256, 0, st>>>(p->inst.F[p->par][c], fields[c], p->inst);
  }
  RFXB_CUDA(cudaGetLastError());
  return 0;
}

int rfxb_plan_store_fields(RfxbPlan* p, float* const* fields, void* stream) {
  if (!p || !fields) return fail(RFXB_E_INVALID, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const long long cells = (long long)p->nx * p->ny * p->nz;
  const int blocks = (int)std::min<long long>((cells + 255) / 256, 65535LL * 8);
  for (int c = 0; c < 6; ++c) {
    if (!fields[c]) return fail(RFXB_E_INVALID, "null field pointer");
    unpack_kernel<<<blocks, 256, 0, st>>>(fields[c], p->inst.F[p->par][c], p->inst);
  }
  RFXB_CUDA(cudaGetLastError());
  return 0;
}

int rfxb_plan_advance(RfxbPlan* p, const RfxbStepIO* io, int step0, int n_steps, void* stream) {
  if (!p) return fail(RFXB_E_INVALID, "null plan");
  return group_advance(p->self_group, io, step0, n_steps, static_cast<cudaStream_t>(stream));
}

int rfxb_forward(RfxbPlan* p, const RfxbStepIO* io, float* const* fields, int step0, int n_steps, void* stream) {
  if (int rc = rfxb_plan_load_fields(p, fields, stream)) return rc;
  if (int rc = rfxb_plan_advance(p, io, step0, n_steps, stream)) return rc;
  return rfxb_plan_store_fields(p, fields, stream);
}

int rfxb_plan_record_history(RfxbPlan* p, int step0, int n_steps) {
  if (!p) return fail(RFXB_E_INVALID, "null plan");
  if (p->hcells == 0) return fail(RFXB_E_STATE, "plan has no gradient region");
  if (n_steps < 0 || step0 < 0) return fail(RFXB_E_INVALID, "negative history range");
  const long long need = (long long)n_steps * 6 * p->hcells;
  if (need > p->hist_cap) {
    cudaDeviceSynchronize();
    if (p->hist) {
      auto it = std::find(p->allocs.begin(), p->allocs.end(), (void*)p->hist);
      if (it != p->allocs.end()) p->allocs.erase(it);
      cudaFree(p->hist);
      p->hist = nullptr;
    }
    if (int rc = p->alloc(&p->hist, need)) return rc;
    p->hist_cap = need;
  }
  p->inst.hist = p->hist;
  p->inst.hist_ld = 6 * p->hcells;
  p->inst.hist_step0 = step0;
  p->inst.hist_nsteps = n_steps;
  return 0;
}

int rfxb_plan_checkpoint_reserve(RfxbPlan* p, int n_slots) {
  if (!p || n_slots < 0) return fail(RFXB_E_INVALID, "bad checkpoint request");
  const long long per = 6 * p->elems + 2 * (p->psi_elems[0] + p->psi_elems[1] + p->psi_elems[2]);
  while ((int)p->ckpt.size() < n_slots) {
    float* q = nullptr;
    if (int rc = p->alloc(&q, per)) return rc;
    p->ckpt.push_back(q);
    p->ckpt_valid.push_back(0);
  }
  return 0;
}

int rfxb_plan_checkpoint_save(RfxbPlan* p, int slot, void* stream) {
  if (!p || slot < 0 || slot >= (int)p->ckpt.size()) return fail(RFXB_E_INVALID, "checkpoint slot out of range");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  float* dst = p->ckpt[slot];
  for (int c = 0; c < 6; ++c) {
    RFXB_CUDA(cudaMemcpyAsync(dst, p->inst.F[p->par][c], p->elems * sizeof(float), cudaMemcpyDeviceToDevice, st));
    dst += p->elems;
  }
  for (int a = 0; a < 3; ++a) {
    if (p->psi_elems[a] == 0) continue;
    RFXB_CUDA(cudaMemcpyAsync(dst, p->inst.psH[p->ppar][a], p->psi_elems[a] * sizeof(float), cudaMemcpyDeviceToDevice, st));
    dst += p->psi_elems[a];
    RFXB_CUDA(cudaMemcpyAsync(dst, p->inst.psE[p->ppar][a], p->psi_elems[a] * sizeof(float), cudaMemcpyDeviceToDevice, st));
    dst += p->psi_elems[a];
  }
  p->ckpt_valid[slot] = 1;
  return 0;
}

int rfxb_plan_checkpoint_load(RfxbPlan* p, int slot, void* stream) {
  if (!p || slot < 0 || slot >= (int)p->ckpt.size()) return fail(RFXB_E_INVALID, "checkpoint slot out of range");
  if (!p->ckpt_valid[slot]) return fail(RFXB_E_STATE, "checkpoint slot was never saved");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const float* src = p->ckpt[slot];
  for (int c = 0; c < 6; ++c) {
    RFXB_CUDA(cudaMemcpyAsync(p->inst.F[p->par][c], src, p->elems * sizeof(float), cudaMemcpyDeviceToDevice, st));
    src += p->elems;
  }
  for (int a = 0; a < 3; ++a) {
    if (p->psi_elems[a] == 0) continue;
    RFXB_CUDA(cudaMemcpyAsync(p->inst.psH[p->ppar][a], src, p->psi_elems[a] * sizeof(float), cudaMemcpyDeviceToDevice, st));
    src += p->psi_elems[a];
    RFXB_CUDA(cudaMemcpyAsync(p->inst.psE[p->ppar][a], src, p->psi_elems[a] * sizeof(float), cudaMemcpyDeviceToDevice, st));
    src += p->psi_elems[a];
  }
  return 0;
}

namespace {
struct StateHeader {          // leading 128 bytes of a state blob
  char magic[8];
  int nx, ny, nz, ncp;
  unsigned cpml_axes, n_dft;
  long long elems, psi_elems[3], dft_bytes, total;
  char pad[128 - 8 - 6 * 4 - 6 * 8];
};
static_assert(sizeof(StateHeader) == 128, "state header is 128 bytes");
const char kStateMagic[8] = {'R', 'F', 'X', 'B', 'S', 'T', '0', '1'};

StateHeader state_header(const RfxbPlan* p) {
  StateHeader h{};
  std::memcpy(h.magic, kStateMagic, 8);
  h.nx = p->nx; h.ny = p->ny; h.nz = p->nz;
  h.ncp = p->inst.ncp;
  h.cpml_axes = p->inst.cpml_axes;
  h.n_dft = (unsigned)p->dft.size();
  h.elems = p->elems;
  for (int a = 0; a < 3; ++a) h.psi_elems[a] = p->psi_elems[a];
  h.dft_bytes = 0;
  for (size_t q = 0; q < p->dft.size(); ++q) h.dft_bytes += p->dft[q].n_freqs * p->dft_cells[q] * (long long)sizeof(float2);
  long long n = (long long)sizeof(StateHeader) + 6 * p->elems * (long long)sizeof(float);
  for (int a = 0; a < 3; ++a) n += 2 * p->psi_elems[a] * (long long)sizeof(float);
  h.total = n + h.dft_bytes;
  return h;
}

// Sections of the blob after the header, in order: (plan buffer, bytes).
std::vector<std::pair<void*, long long>> state_sections(RfxbPlan* p) {
  std::vector<std::pair<void*, long long>> v;
  for (int c = 0; c < 6; ++c) v.emplace_back(p->inst.F[p->par][c], p->elems * (long long)sizeof(float));
  for (int a = 0; a < 3; ++a) {
    if (p->psi_elems[a] == 0) continue;
    v.emplace_back(p->inst.psH[p->ppar][a], p->psi_elems[a] * (long long)sizeof(float));
    v.emplace_back(p->inst.psE[p->ppar][a], p->psi_elems[a] * (long long)sizeof(float));
  }
  for (size_t q = 0; q < p->dft_cmp.size(); ++q)
    v.emplace_back(p->dft_cmp[q], p->dft[q].n_freqs * p->dft_cells[q] * (long long)sizeof(float2));
  return v;
}
}  // namespace

long long rfxb_plan_state_bytes(const RfxbPlan* p) {
  if (!p) return fail(RFXB_E_INVALID, "null plan");
  return state_header(p).total;
}

int rfxb_plan_save_state(RfxbPlan* p, void* dst, void* stream) {
  if (!p || !dst) return fail(RFXB_E_INVALID, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  const StateHeader h = state_header(p);
  char* out = static_cast<char*>(dst);
  // pageable source: the copy stages the header before returning
  RFXB_CUDA(cudaMemcpyAsync(out, &h, sizeof(h), cudaMemcpyDefault, st));
  RFXB_CUDA(cudaStreamSynchronize(st));
  long long o = sizeof(h);
  for (auto& sec : state_sections(p)) {
    RFXB_CUDA(cudaMemcpyAsync(out + o, sec.first, sec.second, cudaMemcpyDefault, st));
    o += sec.second;
  }
  return 0;
}

int rfxb_plan_restore_state(RfxbPlan* p, const void* src, void* stream) {
  if (!p || !src) return fail(RFXB_E_INVALID, "null argument");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  StateHeader h{};
  RFXB_CUDA(cudaMemcpyAsync(&h, src, sizeof(h), cudaMemcpyDefault, st));
  RFXB_CUDA(cudaStreamSynchronize(st));
  if (std::memcmp(h.magic, kStateMagic, 8) != 0) return fail(RFXB_E_INVALID, "not a plan state blob");
  const StateHeader mine = state_header(p);
  if (h.nx != mine.nx || h.ny != mine.ny || h.nz != mine.nz || h.ncp != mine.ncp ||
      h.cpml_axes != mine.cpml_axes || h.n_dft != mine.n_dft || h.elems != mine.elems ||
      h.psi_elems[0] != mine.psi_elems[0] || h.psi_elems[1] != mine.psi_elems[1] ||
      h.psi_elems[2] != mine.psi_elems[2] || h.dft_bytes != mine.dft_bytes || h.total != mine.total)
    return fail(RFXB_E_SHAPE, "state blob was saved from a plan of another shape, CPML or DFT set-up");
  const char* in = static_cast<const char*>(src);
  long long o = sizeof(h);
  for (auto& sec : state_sections(p)) {
    RFXB_CUDA(cudaMemcpyAsync(sec.first, in + o, sec.second, cudaMemcpyDefault, st));
    o += sec.second;
  }
  return 0;
}

int rfxb_plan_adjoint_begin(RfxbPlan* p, const RfxbAdjointIO* aio, int n_total, void* stream) {
  if (!p || !aio) return fail(RFXB_E_INVALID, "null argument");
  return group_adjoint_begin(p->self_group, aio, n_total, static_cast<cudaStream_t>(stream));
}

int rfxb_plan_adjoint_advance(RfxbPlan* p, const RfxbAdjointIO* aio, int step_hi, int n_steps, void* stream) {
  if (!p || !aio) return fail(RFXB_E_INVALID, "null argument");
  return group_adjoint_advance(p->self_group, aio, step_hi, n_steps, static_cast<cudaStream_t>(stream));
}

int rfxb_batch_create(RfxbPlan* const* plans, int n_plans, RfxbBatch** out) {
  if (!plans || n_plans < 1 || !out) return fail(RFXB_E_INVALID, "bad batch arguments");
  *out = nullptr;
  RfxbBatch* g = new RfxbBatch();
  for (int q = 0; q < n_plans; ++q) {
    if (!plans[q]) { delete g; return fail(RFXB_E_INVALID, "null plan in batch"); }
    g->plans.push_back(plans[q]);
  }
  if (int rc = build_group(g)) { delete g; return rc; }
  *out = g;
  return 0;
}

void rfxb_batch_destroy(RfxbBatch* g) {
  if (!g) return;
  cudaDeviceSynchronize();
  delete g;
}

int rfxb_batch_advance(RfxbBatch* g, const RfxbStepIO* ios, int step0, int n_steps, void* stream) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  return group_advance(g, ios, step0, n_steps, static_cast<cudaStream_t>(stream));
}

int rfxb_batch_record_history(RfxbBatch* g, int step0, int n_steps) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  for (auto* p : g->plans)
    if (p->hcells > 0)
      if (int rc = rfxb_plan_record_history(p, step0, n_steps)) return rc;
  return 0;
}

int rfxb_batch_adjoint_begin(RfxbBatch* g, const RfxbAdjointIO* aios, int n_total, void* stream) {
  if (!g || !aios) return fail(RFXB_E_INVALID, "null argument");
  return group_adjoint_begin(g, aios, n_total, static_cast<cudaStream_t>(stream));
}

int rfxb_batch_adjoint_advance(RfxbBatch* g, const RfxbAdjointIO* aios, int step_hi, int n_steps, void* stream) {
  if (!g || !aios) return fail(RFXB_E_INVALID, "null argument");
  return group_adjoint_advance(g, aios, step_hi, n_steps, static_cast<cudaStream_t>(stream));
}

int rfxb_plan_device_status(RfxbPlan* p, void* stream) {
  if (!p) return fail(RFXB_E_INVALID, "null plan");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RFXB_CUDA(cudaStreamSynchronize(st));
  int v = 0;
  RFXB_CUDA(cudaMemcpy(&v, p->self_group->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (v & 1) return fail(RFXB_E_TIMEOUT, "a pipeline wait in a step kernel ran out (device status word set)");
  if (v & 2) return fail(RFXB_E_WORK, "a persistent step kernel met an invalid work item and skipped it");
  return 0;
}

int rfxb_batch_device_status(RfxbBatch* g, void* stream) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RFXB_CUDA(cudaStreamSynchronize(st));
  int v = 0;
  RFXB_CUDA(cudaMemcpy(&v, g->d_status, sizeof(int), cudaMemcpyDeviceToHost));
  if (v & 1) return fail(RFXB_E_TIMEOUT, "a pipeline wait in a step kernel ran out (device status word set)");
  if (v & 2) return fail(RFXB_E_WORK, "a persistent step kernel met an invalid work item and skipped it");
  return 0;
}

namespace {
int box_energy(RfxbPlan* p, const int* b, const double* wx, const double* wy, const double* wz, double* out,
               void* stream) {
  if (!p || !b || !out) return fail(RFXB_E_INVALID, "plan, box and output are required");
  if (b[0] < 0 || b[1] > p->nx || b[2] < 0 || b[3] > p->ny || b[4] < 0 || b[5] > p->nz || b[0] >= b[1] ||
      b[2] >= b[3] || b[4] >= b[5])
    return fail(RFXB_E_INVALID, "energy box out of range or empty");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RFXB_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
  const long long cells = (long long)(b[1] - b[0]) * (b[3] - b[2]) * (b[5] - b[4]);
  const int blocks = (int)std::max<long long>(1, std::min<long long>((cells + 255) / 256, 8LL * sm_count()));
  box_energy_kernel<<<blocks, 256, 0, st>>>(p->inst, p->par, b[0], b[1], b[2], b[3], b[4], b[5], wx, wy, wz, out);
  RFXB_CUDA(cudaGetLastError());
  return 0;
}
}  // namespace

int rfxb_plan_box_energy(RfxbPlan* p, const int* b, double* out, void* stream) {
  return box_energy(p, b, nullptr, nullptr, nullptr, out, stream);
}

int rfxb_plan_box_energy_weighted(RfxbPlan* p, const int* b, const double* wx_dev, const double* wy_dev,
                                  const double* wz_dev, double* out, void* stream) {
  if (!wx_dev || !wy_dev || !wz_dev) return fail(RFXB_E_INVALID, "the three weight tables are required");
  return box_energy(p, b, wx_dev, wy_dev, wz_dev, out, stream);
}

int rfxb_plan_box_flux(RfxbPlan* p, const int* b, double* out, void* stream) {
  if (!p || !b || !out) return fail(RFXB_E_INVALID, "plan, box and output are required");
  if (b[0] < 0 || b[1] >= p->nx || b[2] < 0 || b[3] >= p->ny || b[4] < 0 || b[5] >= p->nz || b[0] >= b[1] ||
      b[2] >= b[3] || b[4] >= b[5])
    return fail(RFXB_E_INVALID, "flux box out of range or empty");
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  RFXB_CUDA(cudaMemsetAsync(out, 0, sizeof(double), st));
  const long long cells = 2LL * ((long long)(b[3] - b[2]) * (b[5] - b[4]) + (long long)(b[1] - b[0]) * (b[5] - b[4]) +
                                 (long long)(b[1] - b[0]) * (b[3] - b[2]));
  const int blocks = (int)std::max<long long>(1, std::min<long long>((cells + 255) / 256, 8LL * sm_count()));
  box_flux_kernel<<<blocks, 256, 0, st>>>(p->inst, p->par, b[0], b[1], b[2], b[3], b[4], b[5], out);
  RFXB_CUDA(cudaGetLastError());
  return 0;
}

int rfxb_plan_forward_variant(const RfxbPlan* p) {
  if (!p || !p->self_group) return -1;
  return p->self_group->fwd_mode;
}

int rfxb_batch_forward_variant(const RfxbBatch* g) {
  if (!g) return -1;
  return g->fwd_mode;
}

namespace {
void step_launches(const RfxbBatch* g, int* fwd, int* rev) {
  if (fwd) {
    if (two_step(g)) *fwd = 1 + 2 * ((g->n_wd1 > 0 ? 1 : 0) + (g->n_wd2 > 0 ? 1 : 0));   // per pass of two steps
    else *fwd = (g->fwd_persist > 0 && g->fwd_split_avail) ? 1 : g->fwd_split ? 2 : 1;
  }
  if (rev) {
    if (g->adj_mode < 0) *rev = -1;
    else if (use_twopass()) *rev = 2;
    else if (g->adj_persist && g->adj_mode == 2 && adj_persist_avail(g)) *rev = 1;
    else if (g->adj_split && g->adj_mode != 0)
      *rev = ((g->adj_lite && g->adj_mode == 2) ? (g->n_wa2y > 0 ? 3 : 2) : 2) - (g->n_wa1 > 0 ? 0 : 1);
    else *rev = 1;
  }
}
}  // namespace

int rfxb_plan_step_launches(const RfxbPlan* p, int* fwd, int* rev) {
  if (!p || !p->self_group) return fail(RFXB_E_INVALID, "null plan");
  step_launches(p->self_group, fwd, rev);
  return 0;
}

int rfxb_batch_step_launches(const RfxbBatch* g, int* fwd, int* rev) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  step_launches(g, fwd, rev);
  return 0;
}

namespace {
void launch_config(const RfxbBatch* g, RfxbLaunchConfig* cur, RfxbLaunchConfig* lim) {
  if (cur)
    *cur = RfxbLaunchConfig{g->fwd_split ? 1 : 0, g->fwd_order, g->adj_lite ? 1 : 0, g->adj_order, g->fwd_persist,
                            g->adj_persist, g->plans[0]->l2promo, g->fwd_depth};
  if (lim)
    *lim = RfxbLaunchConfig{g->fwd_split_avail ? 1 : 0, g->fwd_split_avail ? 1 : 0, g->adj_lite_avail ? 1 : 0,
                            g->adj_split ? 5 : 0, g->fwd_split_avail ? 3 : 0, adj_persist_avail(g) ? 1 : 0, 3, g->fwd_depth_avail ? 2 : 1};
}

int set_launch_config(RfxbBatch* g, const RfxbLaunchConfig* c) {
  if (!c) return fail(RFXB_E_INVALID, "null launch configuration");
  RfxbLaunchConfig lim;
  launch_config(g, nullptr, &lim);
  auto in = [](int v, int hi) { return v >= 0 && v <= hi; };
  if (!in(c->fwd_split, lim.fwd_split) || !in(c->fwd_order, lim.fwd_order) || !in(c->adj_lite, lim.adj_lite) ||
      !in(c->adj_order, lim.adj_order) || !in(c->fwd_persist, lim.fwd_persist) ||
      !in(c->adj_persist, lim.adj_persist) || !in(c->l2_promo, lim.l2_promo) || !in(c->fwd_depth, lim.fwd_depth))
    return fail(RFXB_E_INVALID, "launch configuration outside the limits of this plan/batch");
  if (c->fwd_depth == 2 && c->fwd_persist > 0)
    return fail(RFXB_E_INVALID, "two-step passes and persistent forward launches exclude each other");
  if (c->fwd_depth == 2)
    for (auto* p : g->plans)
      if (int rc = ensure_mid(p)) return rc;
  // cached graphs hold the old launch sequence: drop them once nothing runs
  RFXB_CUDA(cudaDeviceSynchronize());
  for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second);
  g->graphs.clear();
  g->graph_use.clear();
  g->fwd_split = c->fwd_split != 0;
  g->fwd_order = c->fwd_order;
  g->adj_lite = c->adj_lite != 0;
  g->adj_order = c->adj_order;
  g->fwd_persist = c->fwd_persist;
  g->adj_persist = c->adj_persist;
  g->fwd_depth = c->fwd_depth == 2 ? 2 : 1;
  for (auto* p : g->plans)
    if (p->l2promo != c->l2_promo) {
      p->l2promo = c->l2_promo;
      if (int rc = reencode_maps(p)) return rc;
    }
  return 0;
}

int debug_fault(RfxbBatch* g, int cta, int wait_limit) {
  if (wait_limit < 1) return fail(RFXB_E_INVALID, "wait_limit must be >= 1");
  RFXB_CUDA(cudaDeviceSynchronize());
  for (auto& kv : g->graphs) cudaGraphExecDestroy(kv.second);
  g->graphs.clear();
  g->graph_use.clear();
  g->fault_cta = cta;
  g->wait_limit = wait_limit;
  return 0;
}

int debug_poison(RfxbBatch* g, int list, int index) {
  RfxbWork* lists[5] = {g->d_wf2, g->d_wf1, g->d_wa2y, g->d_wa4, g->d_wa1};
  const int counts[5] = {g->n_wf2, g->n_wf1, g->n_wa2y, g->n_wa4, g->n_wa1};
  if (list < 0 || list > 4 || !lists[list] || index < 0 || index >= counts[list])
    return fail(RFXB_E_INVALID, "no such work list entry");
  RFXB_CUDA(cudaDeviceSynchronize());
  RfxbWork w{};
  RFXB_CUDA(cudaMemcpy(&w, lists[list] + index, sizeof(w), cudaMemcpyDeviceToHost));
  w.xb = w.xa;   // an empty x range: outside every kernel's contract
  RFXB_CUDA(cudaMemcpy(lists[list] + index, &w, sizeof(w), cudaMemcpyHostToDevice));
  return 0;
}
}  // namespace

int rfxb_batch_debug_fault(RfxbBatch* g, int cta, int wait_limit) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  return debug_fault(g, cta, wait_limit);
}

int rfxb_batch_debug_poison(RfxbBatch* g, int list, int index) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  return debug_poison(g, list, index);
}

int rfxb_plan_launch_config(const RfxbPlan* p, RfxbLaunchConfig* current, RfxbLaunchConfig* limits) {
  if (!p || !p->self_group) return fail(RFXB_E_INVALID, "null plan");
  launch_config(p->self_group, current, limits);
  return 0;
}

int rfxb_plan_set_launch_config(RfxbPlan* p, const RfxbLaunchConfig* config) {
  if (!p || !p->self_group) return fail(RFXB_E_INVALID, "null plan");
  return set_launch_config(p->self_group, config);
}

int rfxb_batch_launch_config(const RfxbBatch* g, RfxbLaunchConfig* current, RfxbLaunchConfig* limits) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  launch_config(g, current, limits);
  return 0;
}

int rfxb_batch_set_launch_config(RfxbBatch* g, const RfxbLaunchConfig* config) {
  if (!g) return fail(RFXB_E_INVALID, "null batch");
  return set_launch_config(g, config);
}

int rfxb_debug_work_lists(int n_plans, const int32_t* dims, int32_t resident, int32_t which, int32_t* out,
                          int32_t cap, int32_t* n_out) {
  if (n_plans <= 0 || !dims || resident <= 0 || which < 0 || which > 9 || !n_out)
    return fail(RFXB_E_INVALID, "rfxb_debug_work_lists: bad arguments");
  std::vector<std::unique_ptr<RfxbPlan>> own;
  std::vector<RfxbPlan*> plans;
  for (int q = 0; q < n_plans; ++q) {
    const int32_t* d = dims + 5 * q;
    if (d[0] < 2 || d[1] < 2 || d[2] < 2 || d[3] < 0 || d[4] < 0 || d[4] > 7)
      return fail(RFXB_E_INVALID, "rfxb_debug_work_lists: bad plan dims");
    auto p = std::make_unique<RfxbPlan>();
    p->nx = d[0];
    p->ny = d[1];
    p->nz = d[2];
    p->inst.ncp = d[3];
    p->inst.cpml_axes = (unsigned)d[4];
    plans.push_back(p.get());
    own.push_back(std::move(p));
  }
  const double slab = slab_weight();
  std::vector<RfxbWork> w;
  if (which == 0) {
    make_balanced_work(plans, resident, slab, 3.0, w);
  } else if (which <= 2) {
    std::vector<WorkSeg> plain, cpml;
    split_segments(plans, slab, plain, cpml);
    balance_segments(which == 1 ? plain : cpml, resident, 3.0, w);
  } else if (which <= 4) {
    std::vector<WorkSeg> plain, cpml;
    split_adj_segments(plans, slab, plain, cpml);
    balance_segments(which == 3 ? plain : cpml, resident, 3.0, w);
  } else if (which <= 6) {
    std::vector<WorkSeg> plain, ys, noy;
    split_adj_segments(plans, slab, plain, ys, &noy);
    balance_segments(which == 5 ? ys : noy, resident, 3.0, w);
  } else {
    std::vector<WorkSeg> d2, plain, cpml;
    split_depth2_segments(plans, slab, d2, plain, cpml);
    balance_segments(which == 7 ? d2 : which == 8 ? plain : cpml, resident, 3.0, w);
    if (which == 7)   // the intermediate-store flags ride in bits 16.. of the plan index
      for (RfxbWork& it : w) {
        const int mid = depth2_mid_flags(*plans[it.inst], it);
        it.inst |= mid << 16;
      }
  }
  *n_out = (int32_t)w.size();
  if (!out) return 0;
  if (cap < (int32_t)w.size()) return fail(RFXB_E_INVALID, "rfxb_debug_work_lists: output capacity too small");
  for (size_t t = 0; t < w.size(); ++t) {
    int32_t* o = out + 5 * t;
    o[0] = w[t].inst;
    o[1] = w[t].y0;
    o[2] = w[t].z0;
    o[3] = w[t].xa;
    o[4] = w[t].xb;
  }
  return 0;
}

int rfxb_plan_adjoint_variant(const RfxbPlan* p) {
  if (!p || !p->self_group) return -1;
  return p->self_group->adj_mode;
}

int rfxb_batch_adjoint_variant(const RfxbBatch* g) {
  if (!g) return -1;
  return g->adj_mode;
}

int64_t rfxb_plan_device_bytes(const RfxbPlan* p) {
  if (!p) return 0;
  int64_t b = 0;
  b += 12 * p->elems * 4;                  // fields
  if (p->mid) b += 6 * p->elems * 4;       // intermediate state of two-step passes
  b += 3 * p->elems * 4;                   // ca cb ce
  if (p->ch) b += p->elems * 4;
  if (p->emask) b += p->elems;
  b += 4 * (p->psi_elems[0] + p->psi_elems[1] + p->psi_elems[2]) * 4;
  if (p->adj_alloc) b += (12 * p->elems + 4 * (p->psi_elems[0] + p->psi_elems[1] + p->psi_elems[2])) * 4;
  b += p->hist_cap * 4;
  b += (int64_t)p->ckpt.size() * (6 * p->elems + 2 * (p->psi_elems[0] + p->psi_elems[1] + p->psi_elems[2])) * 4;
  return b;
}

}  // extern "C"
