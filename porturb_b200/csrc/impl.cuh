// Host-side implementation of one dycore handle for a stencil type R and a
// tracer count NTR.  pu_dycore.cu holds the C entry points; impl_inst.cu is
// compiled once per (R, NTR) with PU_REAL / PU_NTR defined.
#pragma once

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstring>
#include <functional>
#include <string>
#include <type_traits>
#include <vector>

#include <nvtx3/nvToolsExt.h>

#include "../../include/pu_dycore.h"
#include "dycore_kernels.cuh"
#include "learned.cuh"
#include "nccl_dyn.h"

namespace pu {

void set_error(const std::string &msg);

#define PU_CK(x)                                                                          \
  do {                                                                                    \
    cudaError_t e_ = (x);                                                                 \
    if (e_ != cudaSuccess) {                                                              \
      set_error(std::string(#x) + ": " + cudaGetErrorString(e_));                         \
      return PU_ERR_CUDA;                                                                 \
    }                                                                                     \
  } while (0)

#define PU_LAUNCHED()                                                                     \
  do {                                                                                    \
    cudaError_t e_ = cudaGetLastError();                                                  \
    if (e_ != cudaSuccess) {                                                              \
      set_error(std::string("kernel launch: ") + cudaGetErrorString(e_));                 \
      return PU_ERR_CUDA;                                                                 \
    }                                                                                     \
    launches++;                                                                           \
  } while (0)

// A named range for profilers (NVTX; a no-op unless a tool is attached).
struct NvtxRange {
  explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
  ~NvtxRange() { nvtxRangePop(); }
  NvtxRange(const NvtxRange &) = delete;
  NvtxRange &operator=(const NvtxRange &) = delete;
};

#define PU_TRY(x)                 \
  do {                            \
    int rc_ = (x);                \
    if (rc_ != PU_OK) return rc_; \
  } while (0)

// ---------------------------------------------------------------------------
// Domain decomposition (coupler.h:132-229): a handle can be the (px, py) tile
// of an nproc_x x nproc_y grid of tiles over the global domain; the halos
// beyond its x and y edges come from the neighbouring tiles every stage
// (coupler.h:985-1165, dynamics_rk.h:808-912).
// ---------------------------------------------------------------------------
// Buffers of one halo exchange, per direction d = x-, x+, y-, y+: snd[d] holds
// this tile's cells next to edge d, rcv[d] receives the neighbour's cells
// beyond edge d (the neighbour's snd[d ^ 1]).
// hsnd/hrcv: pinned host copies of the slabs for a host transport (made on
// first use).
struct HaloSet {
  void *snd[4] = {nullptr, nullptr, nullptr, nullptr};
  void *rcv[4] = {nullptr, nullptr, nullptr, nullptr};
  void *hsnd[4] = {nullptr, nullptr, nullptr, nullptr};
  void *hrcv[4] = {nullptr, nullptr, nullptr, nullptr};
  size_t bytes[4] = {0, 0, 0, 0};
  void release() {
    for (int d = 0; d < 4; d++) {
      if (snd[d]) cudaFree(snd[d]);
      if (rcv[d]) cudaFree(rcv[d]);
      if (hsnd[d]) cudaFreeHost(hsnd[d]);
      if (hrcv[d]) cudaFreeHost(hrcv[d]);
      snd[d] = rcv[d] = hsnd[d] = hrcv[d] = nullptr;
      bytes[d] = 0;
    }
  }
};

// Width of the immersed-proportion halo gathered at init: the any_immersed10
// flag of a halo cell next to the tile (the centre of the stencils of cells
// -1 and n) looks 10 cells further.
constexpr int INIT_HALO = 12;

struct Decomposition {
  bool on = false;
  pu_decomp d{};
  int rank = 0, nranks = 1;  // rank = py*nproc_x + px (coupler.h:168-171)
  int nbr[4] = {0, 0, 0, 0}; // ranks beyond the x-, x+, y-, y+ edges, periodic (coupler.h:203-214)
  ncclComm_t comm = nullptr; // null: a host transport (below) or an in-process group of tiles (pu_dycore_group_*)
  bool host = false;         // the caller's host transport moves the slabs and sums
  pu_host_transport ht{};
  HaloSet state;             // the stage input's raw state, HALO_W wide
  uint8_t *fslab[4] = {nullptr, nullptr, nullptr, nullptr};  // immersed flags of the cells in state.rcv
  HaloSet ix, iy;            // the immersed proportion at init, INIT_HALO wide (FP64)
  double *dprop = nullptr, *ext_x = nullptr, *ext = nullptr;  // init scratch
};

struct ImplBase {
  pu_config cfg{};
  cudaStream_t st = nullptr;
  int ntr = 0, S = 0, F = 0, nzh = 0;
  size_t N = 0, NP = 0;
  bool inited = false, has_imm = false;
  int imm_kc = 0;   // 1 + the highest level holding an immersed flag (immersed, or one within 10 cells)
  bool owns = true;                           // false: buffers point into caller-provided scratch
  long long launches = 0;
  // Device buffers.
  void *s[3] = {nullptr, nullptr, nullptr};   // state, two stage buffers
  void *txy = nullptr;                        // x/y tendency of the current stage
  double *staging = nullptr;                  // (5+ntr)*N doubles for host-side coupler views
  double *cells = nullptr, *edges = nullptr;  // FP64 profiles [3][nzh], [3][nz+1]
  double *rho_off = nullptr, *rt_off = nullptr;
  void *tabs = nullptr;                       // level tables of type R
  uint8_t *flags = nullptr;
  void *imm_mult = nullptr;
  int *err = nullptr;
  double *sums = nullptr;
  double *diag_part = nullptr, *diag_out = nullptr;
  int diag_blocks = 0;
  // The copy stream and chunk events of the overlapped time_step (created at
  // its first use); a decomposed tile's NCCL exchange runs on the same stream
  // when it overlaps the interior tiles (dec_ev orders it).
  cudaStream_t cs = nullptr;
  std::vector<cudaEvent_t> io_ev;
  cudaEvent_t dec_ev[2] = {nullptr, nullptr};
  // A decomposed stage whose interior tiles already ran: the x/y kernel takes
  // the edge tiles only.
  bool dec_edges_only = false;
  // Event-based per-kernel timing (pu_dycore_profile).
  bool profiling = false;
  std::vector<cudaEvent_t> ev_pool;
  std::vector<std::pair<int, std::pair<cudaEvent_t, cudaEvent_t>>> ev_pairs;
  size_t ev_next = 0;

  cudaEvent_t next_event() {
    if (ev_next == ev_pool.size()) {
      cudaEvent_t e;
      cudaEventCreate(&e);
      ev_pool.push_back(e);
    }
    return ev_pool[ev_next++];
  }
  // Records a start event when profiling; returns it (or null).
  cudaEvent_t prof_begin() {
    if (!profiling) return nullptr;
    cudaEvent_t e = next_event();
    cudaEventRecord(e, st);
    return e;
  }
  void prof_end(int kind, cudaEvent_t start) {
    if (!start) return;
    cudaEvent_t e = next_event();
    cudaEventRecord(e, st);
    ev_pairs.push_back({kind, {start, e}});
  }
  void prof_reset() {
    ev_pairs.clear();
    ev_next = 0;
  }
  int prof_read(pu_profile *out) {
    PU_CK(cudaStreamSynchronize(st));
    for (int q = 0; q < PU_PROFILE_KINDS; q++) {
      out->ms[q] = 0;
      out->launches[q] = 0;
    }
    for (auto &p : ev_pairs) {
      float ms = 0;
      PU_CK(cudaEventElapsedTime(&ms, p.second.first, p.second.second));
      out->ms[p.first] += ms;
      out->launches[p.first]++;
    }
    return PU_OK;
  }

  // Learned weights (pu_dycore_learned_*): FP32 master parameters with Adam
  // moments, their bfloat16-rounded copy, tensor-core fragments, the harvested
  // training set and fallback counters.
  int weno_mode = PU_WENO_PLAIN;
  float ml_jump = 0.5f;   // largest normalised neighbour jump given learned weights
  float *ml_theta = nullptr, *ml_m = nullptr, *ml_v = nullptr, *ml_wq = nullptr, *ml_grad = nullptr;
  float *ml_partial = nullptr;
  int ml_partial_blocks = 0;
  uint32_t *ml_frags = nullptr;
  float *ml_xs = nullptr, *ml_ts = nullptr;
  long ml_n = 0, ml_cap = 0, ml_step = 0;
  bool ml_ready = false;
  unsigned long long *ml_counts = nullptr;   // [0] stencils on the learned path, [1] fallbacks

  int ml_alloc() {
    if (ml_theta) return PU_OK;
    const size_t P = mlp::NPARAM;
    void *p;
    for (float **dst : {&ml_theta, &ml_m, &ml_v, &ml_wq}) {
      PU_CK(cudaMalloc(&p, P * sizeof(float)));
      *dst = static_cast<float *>(p);
    }
    PU_CK(cudaMalloc(&p, (P + 1) * sizeof(float)));
    ml_grad = static_cast<float *>(p);
    PU_CK(cudaMalloc(&p, 32 * mlp::FRAG_WORDS * sizeof(uint32_t)));
    ml_frags = static_cast<uint32_t *>(p);
    PU_CK(cudaMalloc(&p, 2 * sizeof(unsigned long long)));
    ml_counts = static_cast<unsigned long long *>(p);
    PU_CK(cudaMemsetAsync(ml_counts, 0, 2 * sizeof(unsigned long long), st));
    // He-uniform weights and zero biases from splitmix64(seed 0 << 32 | index).
    std::vector<float> h(P, 0.f);
    for (size_t q = 0; q < P; q++) {
      if (mlp::is_bias(int(q))) continue;
      unsigned long long z = q + 0x9E3779B97F4A7C15ull;
      z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
      z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
      z = z ^ (z >> 31);
      const double u = double(z >> 11) * (1.0 / 9007199254740992.0) * 2.0 - 1.0;
      const int fan_in = int(q) < mlp::OFF_B1 ? mlp::NIN : mlp::NH;
      h[q] = float(u * std::sqrt(6.0 / fan_in));
    }
    return ml_set(h.data());
  }

  int ml_set(const float *theta_host) {
    PU_CK(cudaMemcpyAsync(ml_theta, theta_host, mlp::NPARAM * sizeof(float), cudaMemcpyHostToDevice, st));
    PU_CK(cudaMemsetAsync(ml_m, 0, mlp::NPARAM * sizeof(float), st));
    PU_CK(cudaMemsetAsync(ml_v, 0, mlp::NPARAM * sizeof(float), st));
    ml_step = 0;
    return ml_refresh();
  }

  // bfloat16 copy and tensor-core fragments of the current master parameters.
  int ml_refresh() {
    k_mlp_prepare<<<(mlp::NPARAM + 255) / 256, 256, 0, st>>>(ml_theta, ml_wq);
    PU_LAUNCHED();
    k_mlp_frags<<<1, 32, 0, st>>>(ml_theta, ml_frags);
    PU_LAUNCHED();
    ml_ready = true;
    return PU_OK;
  }

  int ml_get(float *theta_host) {
    PU_CK(cudaMemcpyAsync(theta_host, ml_theta, mlp::NPARAM * sizeof(float), cudaMemcpyDeviceToHost, st));
    PU_CK(cudaStreamSynchronize(st));
    return PU_OK;
  }

  int ml_reserve(long n) {
    if (n <= ml_cap) return PU_OK;
    n = std::max(n, 2 * ml_cap);
    void *xs, *ts;
    PU_CK(cudaMalloc(&xs, size_t(n) * 9 * sizeof(float)));
    cudaError_t e = cudaMalloc(&ts, size_t(n) * 5 * sizeof(float));
    if (e != cudaSuccess) {
      cudaFree(xs);
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return PU_ERR_NOMEM;
    }
    if (ml_n) {
      PU_CK(cudaMemcpyAsync(xs, ml_xs, size_t(ml_n) * 9 * sizeof(float), cudaMemcpyDeviceToDevice, st));
      PU_CK(cudaMemcpyAsync(ts, ml_ts, size_t(ml_n) * 5 * sizeof(float), cudaMemcpyDeviceToDevice, st));
      PU_CK(cudaStreamSynchronize(st));
    }
    cudaFree(ml_xs);
    cudaFree(ml_ts);
    ml_xs = static_cast<float *>(xs);
    ml_ts = static_cast<float *>(ts);
    ml_cap = n;
    return PU_OK;
  }

  int ml_partials(int nblocks) {
    if (nblocks <= ml_partial_blocks) return PU_OK;
    cudaFree(ml_partial);
    void *p;
    PU_CK(cudaMalloc(&p, size_t(nblocks) * (mlp::NPARAM + 1) * sizeof(float)));
    ml_partial = static_cast<float *>(p);
    ml_partial_blocks = nblocks;
    return PU_OK;
  }

  // One forward/backward over `batch` samples of (xs, ts): gradient in ml_grad.
  int ml_fwd_bwd(const float *xs, const float *ts, long ndata, int batch, unsigned long long seed, int sequential) {
    const int nb = (batch + mlp::TB - 1) / mlp::TB;
    int rc = ml_partials(nb);
    if (rc) return rc;
    PU_CK(cudaFuncSetAttribute(k_mlp_fwd_bwd, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(mlp_train_smem_bytes())));
    k_mlp_fwd_bwd<<<nb, mlp::TB, mlp_train_smem_bytes(), st>>>(ml_wq, xs, ts, ndata, ml_step, seed, batch, sequential,
                                                               ml_partial);
    PU_LAUNCHED();
    k_mlp_reduce<<<(mlp::NPARAM + 1 + 255) / 256, 256, 0, st>>>(ml_partial, nb, ml_grad);
    PU_LAUNCHED();
    return PU_OK;
  }

  int ml_train(int steps, int batch, double lr, unsigned long long seed, pu_learn_stats *out) {
    if (ml_n <= 0) {
      set_error("no harvested stencils: call pu_dycore_learned_harvest first");
      return PU_ERR_STATE;
    }
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    cudaEventRecord(e0, st);
    float loss0 = 0, loss1 = 0;
    for (int it = 0; it < steps; it++) {
      int rc = ml_fwd_bwd(ml_xs, ml_ts, ml_n, batch, seed, 0);
      if (rc) return rc;
      if (it == 0 || it == steps - 1) {
        float L;
        PU_CK(cudaMemcpyAsync(&L, ml_grad + mlp::NPARAM, sizeof(float), cudaMemcpyDeviceToHost, st));
        PU_CK(cudaStreamSynchronize(st));
        (it == 0 ? loss0 : loss1) = L / batch;
      }
      ml_step++;
      const float b1 = 0.9f, b2 = 0.999f;
      const float bc1 = float(1.0 - std::pow(0.9, double(ml_step))), bc2 = float(1.0 - std::pow(0.999, double(ml_step)));
      k_adam<<<(mlp::NPARAM + 255) / 256, 256, 0, st>>>(ml_theta, ml_m, ml_v, ml_grad, float(lr), b1, b2, 1e-8f, bc1, bc2);
      PU_LAUNCHED();
      k_mlp_prepare<<<(mlp::NPARAM + 255) / 256, 256, 0, st>>>(ml_theta, ml_wq);
      PU_LAUNCHED();
    }
    cudaEventRecord(e1, st);
    PU_CK(cudaEventSynchronize(e1));
    float ms = 0;
    cudaEventElapsedTime(&ms, e0, e1);
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    int rc = ml_refresh();
    if (rc) return rc;
    if (out) {
      out->loss_first = loss0;
      out->loss_last = loss1;
      out->steps = steps;
      out->samples = ml_n;
      out->ms = ms;
    }
    return PU_OK;
  }

  // Check entries: network weights or gradients of host-provided stencils.
  int ml_eval(const float *x, long n, float *wl, float *wr, int use_mma) {
    float *dx, *dl, *dr;
    void *p;
    PU_CK(cudaMalloc(&p, size_t(n) * 19 * sizeof(float)));
    dx = static_cast<float *>(p);
    dl = dx + n * 9;
    dr = dl + n * 5;
    int rc = PU_OK;
    cudaMemcpyAsync(dx, x, size_t(n) * 9 * sizeof(float), cudaMemcpyHostToDevice, st);
    if (use_mma) {
      const int warps = 4;
      k_mlp_eval_mma<<<unsigned((n + 32 * warps - 1) / (32 * warps)), 32 * warps, warps * mlp::WARP_SMEM_BYTES, st>>>(
          ml_frags, dx, n, dl, dr);
    } else {
      k_mlp_eval<<<unsigned((n + 255) / 256), 256, 0, st>>>(ml_wq, dx, n, dl);
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("kernel launch: ") + cudaGetErrorString(e));
      rc = PU_ERR_CUDA;
    } else {
      launches++;
      cudaMemcpyAsync(wl, dl, size_t(n) * 5 * sizeof(float), cudaMemcpyDeviceToHost, st);
      if (use_mma && wr) cudaMemcpyAsync(wr, dr, size_t(n) * 5 * sizeof(float), cudaMemcpyDeviceToHost, st);
      if (cudaStreamSynchronize(st) != cudaSuccess) rc = PU_ERR_CUDA;
    }
    cudaFree(dx);
    return rc;
  }

  int ml_gradient(const float *x, const float *t, long n, float *grad, double *loss) {
    void *p;
    PU_CK(cudaMalloc(&p, size_t(n) * 14 * sizeof(float)));
    float *dx = static_cast<float *>(p), *dt = dx + n * 9;
    cudaMemcpyAsync(dx, x, size_t(n) * 9 * sizeof(float), cudaMemcpyHostToDevice, st);
    cudaMemcpyAsync(dt, t, size_t(n) * 5 * sizeof(float), cudaMemcpyHostToDevice, st);
    int rc = ml_fwd_bwd(dx, dt, n, int(n), 0, 1);
    float h[mlp::NPARAM + 1];
    if (!rc && cudaMemcpyAsync(h, ml_grad, sizeof(h), cudaMemcpyDeviceToHost, st) == cudaSuccess &&
        cudaStreamSynchronize(st) == cudaSuccess) {
      for (int q = 0; q < mlp::NPARAM; q++) grad[q] = h[q];
      if (loss) *loss = double(h[mlp::NPARAM]) / double(n);
    } else if (!rc) {
      rc = PU_ERR_CUDA;
    }
    cudaFree(p);
    return rc;
  }

  virtual int ml_harvest(long n, unsigned long long seed) = 0;

  // ---- decomposition ----
  Decomposition dc;
  bool sim2d() const { return cfg.ny == 1; }
  HaloSet &halo(int which) { return which == 0 ? dc.state : which == 1 ? dc.ix : dc.iy; }
  void dec_release() {
    dc.state.release();
    dc.ix.release();
    dc.iy.release();
    for (auto &f : dc.fslab) {
      if (f) cudaFree(f);
      f = nullptr;
    }
    for (double **p : {&dc.dprop, &dc.ext_x, &dc.ext}) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
    if (dc.comm && nccl().ok) nccl().CommDestroy(dc.comm);
    dc.comm = nullptr;
  }
  int nccl_fail(ncclResult_t r, const char *what) {
    set_error(std::string(what) + ": " + (nccl().ok ? nccl().GetErrorString(r) : "NCCL unavailable"));
    return PU_ERR_CUDA;
  }
  // Posts the exchange of one HaloSet with NCCL on the handle's stream.  Per
  // direction pair the posts are (send snd[lo] to the low neighbour, receive
  // rcv[hi] from the high one, send snd[hi] to the high neighbour, receive
  // rcv[lo] from the low one); NCCL matches the sends and receives between
  // two ranks in the order they are posted, so with one or two tiles across a
  // direction (both neighbours the same rank) every rank's first message to
  // the other is its snd[lo], which the other takes into rcv[hi].
  int nccl_exchange(HaloSet &h, bool x, bool y, cudaStream_t on = nullptr) {
    if (!on) on = st;
    auto &api = nccl();
    if (!api.ok || !dc.comm) {
      set_error("NCCL halo exchange without a communicator");
      return PU_ERR_STATE;
    }
    ncclResult_t r = api.GroupStart();
    if (r != ncclSuccess) return nccl_fail(r, "ncclGroupStart");
    ncclResult_t first = ncclSuccess;
    auto note = [&](ncclResult_t q) {
      if (q != ncclSuccess && first == ncclSuccess) first = q;
    };
    for (int a = 0; a < 2; a++) {
      if ((a == 0 && !x) || (a == 1 && !y)) continue;
      const int lo = 2 * a, hi = lo + 1;
      note(api.Send(h.snd[lo], h.bytes[lo], ncclUint8, dc.nbr[lo], dc.comm, on));
      note(api.Recv(h.rcv[hi], h.bytes[hi], ncclUint8, dc.nbr[hi], dc.comm, on));
      note(api.Send(h.snd[hi], h.bytes[hi], ncclUint8, dc.nbr[hi], dc.comm, on));
      note(api.Recv(h.rcv[lo], h.bytes[lo], ncclUint8, dc.nbr[lo], dc.comm, on));
    }
    r = api.GroupEnd();
    if (first != ncclSuccess) return nccl_fail(first, "ncclSend/ncclRecv");
    if (r != ncclSuccess) return nccl_fail(r, "ncclGroupEnd");
    return PU_OK;
  }
  // The exchange through the caller's host transport: the active slabs to
  // pinned host memory, the transport's exchange, the received slabs back.
  int host_exchange(HaloSet &h, bool x, bool y, const std::function<int()> &interior = nullptr) {
    void *s[4] = {nullptr, nullptr, nullptr, nullptr}, *r[4] = {nullptr, nullptr, nullptr, nullptr};
    size_t b[4] = {0, 0, 0, 0};
    for (int d = 0; d < 4; d++) {
      if ((d < 2 && !x) || (d >= 2 && !y) || !h.bytes[d]) continue;
      if (!h.hsnd[d]) PU_CK(cudaHostAlloc(&h.hsnd[d], h.bytes[d], cudaHostAllocDefault));
      if (!h.hrcv[d]) PU_CK(cudaHostAlloc(&h.hrcv[d], h.bytes[d], cudaHostAllocDefault));
      PU_CK(cudaMemcpyAsync(h.hsnd[d], h.snd[d], h.bytes[d], cudaMemcpyDeviceToHost, st));
      s[d] = h.hsnd[d];
      r[d] = h.hrcv[d];
      b[d] = h.bytes[d];
    }
    if (interior) {
      // The interior tiles compute while the host moves the slabs.
      PU_TRY(dec_events());
      PU_CK(cudaEventRecord(dec_ev[0], st));
      PU_TRY(interior());
      PU_CK(cudaEventSynchronize(dec_ev[0]));
    } else {
      PU_CK(cudaStreamSynchronize(st));
    }
    const int q = dc.ht.exchange(dc.ht.user, s, r, b, dc.nbr);
    if (q != 0) {
      set_error("host transport: exchange returned " + std::to_string(q));
      return PU_ERR_TRANSPORT;
    }
    for (int d = 0; d < 4; d++)
      if (b[d]) PU_CK(cudaMemcpyAsync(h.rcv[d], h.hrcv[d], b[d], cudaMemcpyHostToDevice, st));
    return PU_OK;
  }
  int dec_events() {
    for (auto &e : dec_ev)
      if (!e) PU_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
    return PU_OK;
  }
  // The halo exchange of one HaloSet through this tile's transport.  With
  // `interior`, the work that needs no halo is launched while the slabs
  // cross: NCCL runs on the side stream between two events, the host
  // transport's callback runs while the device computes.
  int exchange(HaloSet &h, bool x, bool y, const std::function<int()> &interior = nullptr) {
    NvtxRange range("pu:halo_exchange");
    if (dc.comm) {
      if (!interior) return nccl_exchange(h, x, y);
      if (!cs) PU_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
      PU_TRY(dec_events());
      PU_CK(cudaEventRecord(dec_ev[0], st));
      PU_CK(cudaStreamWaitEvent(cs, dec_ev[0], 0));
      PU_TRY(nccl_exchange(h, x, y, cs));
      PU_CK(cudaEventRecord(dec_ev[1], cs));
      PU_TRY(interior());
      PU_CK(cudaStreamWaitEvent(st, dec_ev[1], 0));
      return PU_OK;
    }
    if (dc.host) return host_exchange(h, x, y, interior);
    set_error("halo exchange without a transport");
    return PU_ERR_STATE;
  }
  // Sums the 3*nz column sums over all tiles, in place on the device.
  int sum_columns() {
    const size_t n = size_t(3) * cfg.nz;
    if (dc.comm) {
      const ncclResult_t r = nccl().AllReduce(sums, sums, n, ncclFloat64, ncclSum, dc.comm, st);
      if (r != ncclSuccess) return nccl_fail(r, "ncclAllReduce");
      return PU_OK;
    }
    if (!dc.host) {
      set_error("column sums without a transport");
      return PU_ERR_STATE;
    }
    std::vector<double> h(n);
    PU_CK(cudaMemcpyAsync(h.data(), sums, n * sizeof(double), cudaMemcpyDeviceToHost, st));
    PU_CK(cudaStreamSynchronize(st));
    const int q = dc.ht.allreduce_sum_f64(dc.ht.user, h.data(), n);
    if (q != 0) {
      set_error("host transport: allreduce_sum_f64 returned " + std::to_string(q));
      return PU_ERR_TRANSPORT;
    }
    PU_CK(cudaMemcpyAsync(sums, h.data(), n * sizeof(double), cudaMemcpyHostToDevice, st));
    PU_CK(cudaStreamSynchronize(st));
    return PU_OK;
  }
  bool has_transport() const { return dc.comm != nullptr || dc.host; }
  // Type-dependent parts of the decomposed path (Impl).
  virtual int dec_alloc() = 0;
  virtual int dinit_begin(const pu_state_view *v, const double *prop, const double *proj, int mem) = 0;
  virtual int dinit_hydro(const double *global_sums) = 0;
  virtual int dinit_mid() = 0;
  virtual int dinit_end(const pu_state_view *v) = 0;
  virtual int dec_enforce() = 0;
  virtual int dec_pack(int stage) = 0;
  virtual int dec_compute(int stage, double dt, bool last) = 0;

  virtual ~ImplBase() {
    dec_release();
    for (auto e : ev_pool) cudaEventDestroy(e);
    for (auto e : io_ev) cudaEventDestroy(e);
    for (auto e : dec_ev)
      if (e) cudaEventDestroy(e);
    if (cs) cudaStreamDestroy(cs);
    if (owns)
      for (void *q : {(void *)ml_theta, (void *)ml_m, (void *)ml_v, (void *)ml_wq, (void *)ml_grad, (void *)ml_partial,
                      (void *)ml_frags, (void *)ml_xs, (void *)ml_ts, (void *)ml_counts})
        if (q) cudaFree(q);
  }
  virtual int alloc() = 0;
  virtual int init(const pu_state_view *v, const double *prop, int mem, const double *proj = nullptr) = 0;
  virtual int load_state(const pu_state_view *v) = 0;
  virtual int store_state(pu_state_view *v) = 0;
  virtual int advance(double dt, int nsteps) = 0;
  // time_step (dynamics_rk.h:103-137) after the sub-step count: coupler
  // arrays in, nsteps SSPRK3 steps of dt, coupler arrays out.
  virtual int time_step(pu_state_view *v, double dt, int nsteps) {
    int rc = load_state(v);
    if (!rc) rc = advance(dt, nsteps);
    if (!rc) rc = store_state(v);
    return rc;
  }
  virtual int get_conserved(double *st, double *tr, int mem) = 0;
  virtual int set_conserved(const double *st, const double *tr, int mem) = 0;
  virtual int set_hydrostasis(const double *r, const double *t, const double *p) = 0;
  virtual int diagnostics(pu_diag *out) = 0;
  virtual int perturbations(const pu_state_view *v, double *dens, double *theta, double *press, int mem) = 0;

  int check_err() {
    int h = 0;
    PU_CK(cudaMemcpyAsync(&h, err, sizeof(int), cudaMemcpyDeviceToHost, st));
    PU_CK(cudaStreamSynchronize(st));
    if (h) {
      PU_CK(cudaMemsetAsync(err, 0, sizeof(int), st));
      if (h & ERR_TMA) {
        set_error("a tile copy (TMA) did not complete within its wait limit; the step's results are invalid");
        return PU_ERR_CUDA;
      }
      set_error("the dycore state became non-finite");
      return PU_ERR_NONFINITE;
    }
    return PU_OK;
  }
};

// PU_MEM_AUTO: device (or managed) memory if CUDA knows the pointer as such.
inline int resolve_mem(int mem, const void *p) {
  if (mem != PU_MEM_AUTO) return mem;
  cudaPointerAttributes a;
  if (cudaPointerGetAttributes(&a, p) != cudaSuccess) {
    cudaGetLastError();
    return PU_MEM_HOST;
  }
  return (a.type == cudaMemoryTypeDevice || a.type == cudaMemoryTypeManaged) ? PU_MEM_DEVICE : PU_MEM_HOST;
}

template <class R, int NTR>
struct Impl : ImplBase {
#ifndef PU_XY_TILE_X
#define PU_XY_TILE_X 16
#endif
#ifndef PU_XY_TILE_Y
#define PU_XY_TILE_Y 16
#endif
  static constexpr int XTX_BIG = PU_XY_TILE_X, XTY_BIG = PU_XY_TILE_Y;   // x/y tile for ny >= 16
  static constexpr int LTX = 16, LTY = 16;           // x/y tile of the learned form (ny >= 16)
  static constexpr int XTX_SM = 32, XTY_SM = 4;      // x/y tile for thin domains
  static constexpr int ZT_X = 8, ZT_Z = 32;          // tiled z kernel: columns x levels per block
  static constexpr int ZTX = 32, ZTY = 4;            // z-march columns per block
  LevelTables<R> lt{};
  bool small_tile = false;
  // TMA staging of the tiled z kernel: maps per stage-input buffer s[b]
  // (halo and cell boxes of s[b], the cell boxes of s[0] and txy).
  ZtMaps zt_maps[3];
  bool zt_tma = false;
  // TMA staging of the 16x16 x/y kernel (domains without immersed cells):
  // per stage-input buffer s[b] the interior, halo-row and halo-column boxes.
  XyMaps xy_maps[3];
  bool xy_tma = false;

  // Tensor maps of the state buffers for the tiled z kernel (host-side
  // encoding only, no allocation).  Off when the config asks for thread
  // loads or a buffer breaks a TMA rule.
  void make_maps() {
    zt_tma = false;
    if constexpr (std::is_same<R, float>::value) {
      if (cfg.thread_loads) return;
      const int nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
      bool ok = true;
      for (int b = 0; b < 3 && ok; b++) {
        ok = tma::encode_state(&zt_maps[b].raw, s[b], nx, ny, nz, S, ZT_X, 1, ZT_Z + 10, S) &&
             tma::encode_state(&zt_maps[b].qin, s[b], nx, ny, nz, S, ZT_X, 1, ZT_Z, S) &&
             tma::encode_state(&zt_maps[b].sn, s[0], nx, ny, nz, S, ZT_X, 1, ZT_Z, S) &&
             tma::encode_state(&zt_maps[b].txy, txy, nx, ny, nz, S, ZT_X, 1, ZT_Z, S);
      }
      zt_tma = ok;
      ok = XTX_BIG == 16 && XTY_BIG == 16;
      for (int b = 0; b < 3 && ok; b++) {
        ok = tma::encode_state(&xy_maps[b].in, s[b], nx, ny, nz, S, 16, 16, 1, S) &&
             tma::encode_state(&xy_maps[b].ns, s[b], nx, ny, nz, S, 16, 5, 1, S) &&
             tma::encode_state(&xy_maps[b].ew, s[b], nx, ny, nz, S, 8, 16, 1, S);
      }
      xy_tma = ok;
    }
  }

  ~Impl() override {
    if (!owns) return;
    for (auto p : {s[0], s[1], s[2], txy, (void *)staging, (void *)cells, (void *)edges, (void *)rho_off,
                   (void *)rt_off, tabs, (void *)flags, imm_mult, (void *)err, (void *)sums, (void *)diag_part,
                   (void *)diag_out})
      if (p) cudaFree(p);
  }

  template <class T>
  int dalloc(T *&p, size_t n) {
    void *q = nullptr;
    cudaError_t e = cudaMalloc(&q, n * sizeof(T) > 0 ? n * sizeof(T) : 16);
    if (e != cudaSuccess) {
      set_error(std::string("cudaMalloc: ") + cudaGetErrorString(e));
      return e == cudaErrorMemoryAllocation ? PU_ERR_NOMEM : PU_ERR_CUDA;
    }
    p = static_cast<T *>(q);
    return PU_OK;
  }


  int alloc() override {
    F = 6 + NTR;
    S = 5 + NTR;
    for (int b = 0; b < 3; b++) {
      R *p;
      PU_TRY(dalloc(p, size_t(S) * N));
      s[b] = p;
    }
    R *t;
    PU_TRY(dalloc(t, size_t(S) * N));
    txy = t;
    PU_TRY(dalloc(staging, size_t(5 + NTR) * N));
    PU_TRY(dalloc(cells, size_t(3) * nzh));
    PU_TRY(dalloc(edges, size_t(3) * (cfg.nz + 1)));
    PU_TRY(dalloc(rho_off, size_t(cfg.nz)));
    PU_TRY(dalloc(rt_off, size_t(cfg.nz)));
    R *tb;
    const size_t ntab = 5 * size_t(nzh) + 2 * size_t(cfg.nz + 1) + size_t(cfg.nz);
    PU_TRY(dalloc(tb, ntab));
    tabs = tb;
    lt.rho_h = tb;
    lt.theta_h = tb + nzh;
    lt.rt_inv = tb + 2 * nzh;
    lt.p0_h = tb + 3 * nzh;
    lt.dp_h = tb + 4 * nzh;
    lt.rho_e = tb + 5 * nzh;
    lt.theta_e = lt.rho_e + (cfg.nz + 1);
    lt.rt_target = lt.theta_e + (cfg.nz + 1);
    PU_TRY(dalloc(err, 1));
    PU_CK(cudaMemsetAsync(err, 0, sizeof(int), st));
    PU_TRY(dalloc(sums, size_t(3) * cfg.nz));
    diag_blocks = 296;
    PU_TRY(dalloc(diag_part, size_t(diag_blocks) * NDIAG * 2));
    PU_TRY(dalloc(diag_out, size_t(NDIAG)));
    make_maps();
    return configure();
  }

  // Kernel attributes (no allocation).
  int configure() {
    small_tile = cfg.ny < 16;
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_BIG, XTY_BIG, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_BIG, XTY_BIG, false>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_BIG, XTY_BIG, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_BIG, XTY_BIG, true>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_SM, XTY_SM, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_SM, XTY_SM, false>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_SM, XTY_SM, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_SM, XTY_SM, true>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_BIG, XTY_BIG, false, false, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_BIG, XTY_BIG, false>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_BIG, XTY_BIG, true, false, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_BIG, XTY_BIG, true>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_SM, XTY_SM, false, false, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_SM, XTY_SM, false>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_SM, XTY_SM, true, false, true>,
                               cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(XYShape<R, NTR, XTX_SM, XTY_SM, true>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_z<R, NTR, ZTX, ZTY, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(ZShape<R, NTR, ZTX, ZTY>::bytes)));
    PU_CK(cudaFuncSetAttribute(k_z<R, NTR, ZTX, ZTY, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                               int(ZShape<R, NTR, ZTX, ZTY>::bytes)));
    if constexpr (std::is_same<R, float>::value) {
      PU_CK(cudaFuncSetAttribute(k_zt<NTR, ZT_X, ZT_Z, false>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(ZTShape<NTR, ZT_X, ZT_Z, false>::bytes)));
      PU_CK(cudaFuncSetAttribute(k_zt<NTR, ZT_X, ZT_Z, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(ZTShape<NTR, ZT_X, ZT_Z, true>::bytes)));
      PU_CK(cudaFuncSetAttribute(k_zt<NTR, ZT_X, ZT_Z, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(ZTShape<NTR, ZT_X, ZT_Z, false>::tma_bytes)));
      PU_CK(cudaFuncSetAttribute(k_zt<NTR, ZT_X, ZT_Z, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(ZTShape<NTR, ZT_X, ZT_Z, true>::tma_bytes)));
      if constexpr (XYShape<R, NTR, XTX_BIG, XTY_BIG, false>::TMA_FITS)
        PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_BIG, XTY_BIG, false, false, false, true>,
                                   cudaFuncAttributeMaxDynamicSharedMemorySize,
                                   int(XYShape<R, NTR, XTX_BIG, XTY_BIG, false>::tma_bytes)));
      PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, LTX, LTY, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(XYShape<R, NTR, LTX, LTY, false, true>::bytes)));
      PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, LTX, LTY, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(XYShape<R, NTR, LTX, LTY, true, true>::bytes)));
      PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_SM, XTY_SM, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(XYShape<R, NTR, XTX_SM, XTY_SM, false, true>::bytes)));
      PU_CK(cudaFuncSetAttribute(k_xy<R, NTR, XTX_SM, XTY_SM, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(XYShape<R, NTR, XTX_SM, XTY_SM, true, true>::bytes)));
      PU_CK(cudaFuncSetAttribute(k_z<R, NTR, ZTX, ZTY, false, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(ZShape<R, NTR, ZTX, ZTY, true>::bytes)));
      PU_CK(cudaFuncSetAttribute(k_z<R, NTR, ZTX, ZTY, true, true>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 int(ZShape<R, NTR, ZTX, ZTY, true>::bytes)));
    }
    return PU_OK;
  }

  Thermo thermo() const {
    Thermo th;
    th.R_d = cfg.R_d;
    th.R_v = cfg.R_v;
    th.C0 = cfg.C0;
    th.gamma = cfg.gamma_d;
    th.idWV = cfg.idWV;
    th.adds_mass = 0;
    for (int t = 0; t < NTR; t++)
      if (cfg.tracer_adds_mass[t]) th.adds_mass |= 1u << t;
    return th;
  }

  Grid<R> grid() const {
    Grid<R> G;
    G.nx = cfg.nx;
    G.ny = cfg.ny;
    G.nz = cfg.nz;
    G.N = N;
    G.NP = NP;
    G.rdx = R(1. / cfg.dx);
    G.rdy = R(1. / cfg.dy);
    G.rdz = R(1. / cfg.dz);
    G.bc_x = cfg.bc_x;
    G.bc_y = cfg.bc_y;
    G.bc_z = cfg.bc_z;
    G.sim2d = cfg.ny == 1;
    G.weno_all = cfg.weno_all;
    G.enable_gravity = cfg.enable_gravity;
    G.grav = R(cfg.grav);
    G.fcor = R(2 * 7.2921e-5 * std::sin(cfg.latitude / 180 * M_PI));
    G.gamma = R(cfg.gamma_d);
    {
      double c = 1;
      for (int n = 1; n <= 5; n++) {
        c *= (cfg.gamma_d - (n - 1)) / n;
        G.pc[n - 1] = R(c);
      }
      G.pser = cfg.gamma_d >= 1. && cfg.gamma_d <= 5. / 3.;
    }
    G.tracer_positive = 0;
    for (int t = 0; t < NTR; t++)
      if (cfg.tracer_positive[t]) G.tracer_positive |= 1u << t;
    G.rho_h = lt.rho_h;
    G.theta_h = lt.theta_h;
    G.rt_inv = lt.rt_inv;
    G.p0_h = lt.p0_h;
    G.dp_h = lt.dp_h;
    G.rho_e = lt.rho_e;
    G.theta_e = lt.theta_e;
    G.rt_target = lt.rt_target;
    G.flags = has_imm ? flags : nullptr;
    G.imm_mult = has_imm ? static_cast<const R *>(imm_mult) : nullptr;
    G.hxl = static_cast<const R *>(dc.state.rcv[0]);
    G.hxr = static_cast<const R *>(dc.state.rcv[1]);
    G.hyl = static_cast<const R *>(dc.state.rcv[2]);
    G.hyr = static_cast<const R *>(dc.state.rcv[3]);
    G.fxl = has_imm ? dc.fslab[0] : nullptr;
    G.fxr = has_imm ? dc.fslab[1] : nullptr;
    G.fyl = has_imm ? dc.fslab[2] : nullptr;
    G.fyr = has_imm ? dc.fslab[3] : nullptr;
    G.gx0 = !dc.on || dc.d.px == 0;
    G.gx1 = !dc.on || dc.d.px == dc.d.nproc_x - 1;
    G.gy0 = !dc.on || dc.d.py == 0;
    G.gy1 = !dc.on || dc.d.py == dc.d.nproc_y - 1;
    G.err = err;
    G.k_first = 0;
    G.c_first = 0;
    G.i_first = 0;
    G.j_first = 0;
    G.ml_frags = ml_frags;
    G.ml_counts = ml_counts;
    G.ml_jump = ml_jump;
    return G;
  }

  // Coupler view -> device pointers (copying host arrays into staging).
  int device_view(const pu_state_view *v, CouplerPtrs &cp) {
    const double *src[5] = {v->rho_d, v->uvel, v->vvel, v->wvel, v->temp};
    for (int a = 0; a < 5; a++)
      if (!src[a]) { set_error("coupler view has a null array"); return PU_ERR_INVALID; }
    for (int t = 0; t < NTR; t++)
      if (!v->tracers[t]) { set_error("coupler view has a null tracer array"); return PU_ERR_INVALID; }
    const double *d[5 + NTR];
    if (resolve_mem(v->mem, v->rho_d) == PU_MEM_DEVICE) {
      for (int a = 0; a < 5; a++) d[a] = src[a];
      for (int t = 0; t < NTR; t++) d[5 + t] = v->tracers[t];
    } else {
      for (int a = 0; a < 5 + NTR; a++) {
        const double *h = a < 5 ? src[a] : v->tracers[a - 5];
        PU_CK(cudaMemcpyAsync(staging + size_t(a) * N, h, N * sizeof(double), cudaMemcpyHostToDevice, st));
        d[a] = staging + size_t(a) * N;
      }
    }
    cp.rho_d = d[0]; cp.u = d[1]; cp.v = d[2]; cp.w = d[3]; cp.T = d[4];
    for (int t = 0; t < 8; t++) cp.tr[t] = t < NTR ? d[5 + t] : nullptr;
    return PU_OK;
  }

  unsigned blocks(size_t n, int bs) const { return unsigned((n + bs - 1) / bs); }

  int init(const pu_state_view *v, const double *prop, int mem, const double *proj = nullptr) override {
    if (dc.on) {
      if (!has_transport()) {
        set_error("the tiles of an in-process group are initialised with pu_dycore_group_init");
        return PU_ERR_STATE;
      }
      PU_TRY(dinit_begin(v, prop, proj, mem));
      PU_TRY(sum_columns());
      PU_TRY(dinit_hydro(nullptr));
      PU_TRY(exchange(dc.ix, true, false));
      PU_TRY(dinit_mid());
      if (!sim2d()) PU_TRY(exchange(dc.iy, false, true));
      return dinit_end(v);
    }
    CouplerPtrs cp;
    PU_TRY(device_view(v, cp));
    const Thermo th = thermo();
    k_column_sums<NTR><<<cfg.nz, 256, 0, st>>>(cp, th, cfg.nx, cfg.ny, sums);
    PU_LAUNCHED();
    HydroOut ho{cells, edges, rho_off, rt_off};
    const double r_nx_ny = 1. / (double(cfg.nx) * double(cfg.ny));
    k_hydro_finish<R><<<1, HYDRO_THREADS, 0, st>>>(sums, cfg.nz, r_nx_ny, cfg.gamma_d, cfg.C0, cfg.grav, cfg.dz,
                                       sizeof(R) == 4, ho, lt);
    PU_LAUNCHED();
    // Immersed preprocessing.
    has_imm = false;
    if (prop) {
      double *dprop = nullptr;
      PU_TRY(dalloc(dprop, N));
      if (resolve_mem(mem, prop) == PU_MEM_DEVICE)
        PU_CK(cudaMemcpyAsync(dprop, prop, N * sizeof(double), cudaMemcpyDeviceToDevice, st));
      else PU_CK(cudaMemcpyAsync(dprop, prop, N * sizeof(double), cudaMemcpyHostToDevice, st));
      int rc = PU_OK;
      double *dproj = nullptr;
      if (proj) {
        // The windmill projection weight joins the proportion before the
        // halos, flags and time scales are built (dynamics_rk.h:1019-1025).
        rc = dalloc(dproj, N);
        if (rc == PU_OK) {
          cudaMemcpyAsync(dproj, proj, N * sizeof(double),
                          resolve_mem(mem, proj) == PU_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice,
                          st);
          k_add_inplace<double><<<blocks(N, 256), 256, 0, st>>>(dprop, dproj, N);
          const cudaError_t e = cudaGetLastError();
          if (e != cudaSuccess) {
            set_error(std::string("kernel launch: ") + cudaGetErrorString(e));
            rc = PU_ERR_CUDA;
          } else {
            launches++;
          }
        }
      }
      uint8_t *d0 = nullptr, *d1 = nullptr, *dz = nullptr;
      if (rc == PU_OK) rc = dalloc(d0, N);
      if (rc == PU_OK) rc = dalloc(d1, N);
      if (rc == PU_OK) rc = dalloc(dz, N);
      int *anyp = nullptr;
      if (rc == PU_OK) rc = dalloc(anyp, 1);
      if (rc == PU_OK) rc = imm_prepare(dprop, d0, d1, dz, anyp);
      cudaStreamSynchronize(st);
      for (void *p : {(void *)dprop, (void *)dproj, (void *)d0, (void *)d1, (void *)dz, (void *)anyp})
        if (p) cudaFree(p);
      if (rc != PU_OK) return rc;
    }
    PU_TRY(load_state(v));
    PU_CK(cudaStreamSynchronize(st));
    inited = true;
    return PU_OK;
  }

  int imm_prepare(const double *dprop, uint8_t *a, uint8_t *b, uint8_t *dzero, int *anyp) {
    // Any immersed cell at all?
    PU_CK(cudaMemsetAsync(anyp, 0, sizeof(int), st));
    k_dist_init<<<blocks(N, 256), 256, 0, st>>>(dprop, 0, N, a, 10);
    PU_LAUNCHED();
    // a: distance to immersed (cap 10) -> any_immersed10
    for (int axis = 0; axis < 3; axis++) {
      k_dist_pass<<<blocks(N, 256), 256, 0, st>>>(a, b, cfg.nx, cfg.ny, cfg.nz, axis, 10);
      PU_LAUNCHED();
      std::swap(a, b);
    }
    // dzero: distance to a non-immersed cell (cap 3) -> immersed_tau
    k_dist_init<<<blocks(N, 256), 256, 0, st>>>(dprop, 1, N, dzero, 3);
    PU_LAUNCHED();
    for (int axis = 0; axis < 3; axis++) {
      k_dist_pass<<<blocks(N, 256), 256, 0, st>>>(dzero, b, cfg.nx, cfg.ny, cfg.nz, axis, 3);
      PU_LAUNCHED();
      PU_CK(cudaMemcpyAsync(dzero, b, N, cudaMemcpyDeviceToDevice, st));
    }
    if (!flags) PU_TRY(dalloc(flags, N));
    if (!imm_mult) {
      R *m;
      PU_TRY(dalloc(m, N));
      imm_mult = m;
    }
    k_imm_finish<R><<<blocks(N, 256), 256, 0, st>>>(dprop, a, dzero, cfg.immersed_power, N, flags,
                                                    static_cast<R *>(imm_mult));
    PU_LAUNCHED();
    // has_imm: any flag set (a cell with prop > 0 has distance 0 in `a`).
    std::vector<uint8_t> hf(N);
    PU_CK(cudaMemcpyAsync(hf.data(), flags, N, cudaMemcpyDeviceToHost, st));
    PU_CK(cudaStreamSynchronize(st));
    has_imm = false;
    for (size_t q = 0; q < N && !has_imm; q++) has_imm = (hf[q] & FLAG_IMM) != 0;
    imm_kc = 0;
    for (int k = cfg.nz - 1; k >= 0 && !imm_kc; k--)
      for (size_t q = size_t(k) * NP; q < size_t(k + 1) * NP; q++)
        if (hf[q]) {
          imm_kc = k + 1;
          break;
        }
    return PU_OK;
  }

  int load_state(const pu_state_view *v) override {
    NvtxRange range("pu:load_state");
    CouplerPtrs cp;
    PU_TRY(device_view(v, cp));
    k_load_coupler<R, NTR><<<blocks(N, 256), 256, 0, st>>>(cp, thermo(), rho_off, rt_off, N, NP,
                                                           static_cast<R *>(s[0]), 0, N);
    PU_LAUNCHED();
    return PU_OK;
  }

  int store_state(pu_state_view *v) override {
    NvtxRange range("pu:store_state");
    CouplerOut co;
    double *d[5 + NTR];
    double *dst[5] = {v->rho_d, v->uvel, v->vvel, v->wvel, v->temp};
    for (int a = 0; a < 5; a++)
      if (!dst[a]) { set_error("coupler view has a null array"); return PU_ERR_INVALID; }
    for (int t = 0; t < NTR; t++)
      if (!v->tracers[t]) { set_error("coupler view has a null tracer array"); return PU_ERR_INVALID; }
    const bool on_device = resolve_mem(v->mem, v->rho_d) == PU_MEM_DEVICE;
    for (int a = 0; a < 5 + NTR; a++) {
      double *h = a < 5 ? dst[a] : v->tracers[a - 5];
      d[a] = on_device ? h : staging + size_t(a) * N;
    }
    co.rho_d = d[0]; co.u = d[1]; co.v = d[2]; co.w = d[3]; co.T = d[4];
    for (int t = 0; t < 8; t++) co.tr[t] = t < NTR ? d[5 + t] : nullptr;
    k_store_coupler<R, NTR><<<blocks(N, 256), 256, 0, st>>>(co, thermo(), rho_off, rt_off, N, NP,
                                                            static_cast<const R *>(s[0]), 0, N);
    PU_LAUNCHED();
    if (!on_device)
      for (int a = 0; a < 5 + NTR; a++) {
        double *h = a < 5 ? dst[a] : v->tracers[a - 5];
        PU_CK(cudaMemcpyAsync(h, staging + size_t(a) * N, N * sizeof(double), cudaMemcpyDeviceToHost, st));
      }
    return check_err();
  }

  // Levels from the bottom that take the immersed stage kernels: those an
  // immersed flag reaches (the levels above hold no immersed cell and none
  // within 10 cells, where the immersed code gives the plain code's results);
  // every level for a decomposed tile or when the config asks for it.
  int imm_levels() const { return (dc.on || cfg.imm_all_levels || !has_imm) ? cfg.nz : imm_kc; }

  // The tiled z kernel (k_zt) takes the plain FP32 limiter with weno_all,
  // unless a z chunk was asked for (the march, which gives the same bits).  Its grid has one y row per block
  // row, so ny is held to the grid's y limit.
  bool z_tiled(bool learned) const {
    return std::is_same<R, float>::value && cfg.weno_all && !learned && cfg.z_chunk <= 0 && cfg.ny <= 65535;
  }

  // Learned weights replace the nonlinear limiter where it runs on every
  // stencil (weno_all) in FP32.
  bool learned_active() const {
    return std::is_same<R, float>::value && weno_mode == PU_WENO_LEARNED && ml_ready && cfg.weno_all;
  }

  // The big-tile x/y kernel (no learned weights) on levels [k0, k1): the
  // levels below imm_levels() take the immersed kernel, the others the plain
  // one -- through TMA where the tiles allow it.  b: the index of the stage
  // input among s[] (its tensor maps).
  // Tiles [tx0, tx1) x [ty0, ty1) (all by default).
  template <bool IMM, bool DEC = false>
  int xy_levels(const Grid<R> &G, const R *sin, int b, int k0, int k1, int tx0 = 0, int tx1 = -1, int ty0 = 0,
                int ty1 = -1) {
    using Sh = XYShape<R, NTR, XTX_BIG, XTY_BIG, IMM, false>;
    using Sp = XYShape<R, NTR, XTX_BIG, XTY_BIG, false, false>;
    R *t = static_cast<R *>(txy);
    if (tx1 < 0) tx1 = int(blocks(cfg.nx, XTX_BIG));
    if (ty1 < 0) ty1 = int(blocks(cfg.ny, XTY_BIG));
    if (tx1 <= tx0 || ty1 <= ty0 || k1 <= k0) return PU_OK;
    const int kl = IMM ? std::min(std::max(imm_levels(), k0), k1) : k0;
    const unsigned bx = unsigned(tx1 - tx0), by = unsigned(ty1 - ty0);
    Grid<R> Gt = G;
    Gt.i_first = tx0 * XTX_BIG;
    Gt.j_first = ty0 * XTY_BIG;
    if (kl > k0) {
      Grid<R> Gi = Gt;
      Gi.k_first = k0;
      k_xy<R, NTR, XTX_BIG, XTY_BIG, IMM, false, DEC><<<dim3(bx, by, kl - k0), Sh::NT, Sh::bytes, st>>>(
          Gi, sin, t, xy_maps[b]);
      PU_LAUNCHED();
    }
    if (kl < k1) {
      Grid<R> Gp = Gt;
      Gp.k_first = kl;
      const dim3 g(bx, by, k1 - kl);
      bool staged = false;
      if constexpr (!DEC && Sp::TMA_FITS) {
        if (xy_tma && static_cast<const void *>(sin) == s[b]) {
          k_xy<R, NTR, XTX_BIG, XTY_BIG, false, false, false, true><<<g, Sp::NT, Sp::tma_bytes, st>>>(Gp, sin, t,
                                                                                                    xy_maps[b]);
          staged = true;
        }
      }
      if (!staged)
        k_xy<R, NTR, XTX_BIG, XTY_BIG, false, false, DEC><<<g, Sp::NT, Sp::bytes, st>>>(Gp, sin, t, xy_maps[b]);
      PU_LAUNCHED();
    }
    return PU_OK;
  }

  // The tiled z kernel (FP32, z_tiled) on z chunks [c0, c1) of ZT_Z levels:
  // chunks below ci take the immersed kernel.  Chunk c reads levels
  // 32c-5 .. 32c+36, so it is plain once 32c-5 reaches the first level no
  // flag holds; a periodic z wraps flagged levels into the top chunk, so every
  // chunk stays immersed there.  The maps of this stage input (s[b]); the
  // cell maps of sn and txy are the same for every b.
  template <bool IMM>
  int zt_chunks(const Grid<R> &G, const R *sin, const R *sn, R *sout, R a_n, R a_dt, int n_enforce, int b, int c0,
                int c1) {
    if constexpr (std::is_same<R, float>::value) {
      using Zs = ZTShape<NTR, ZT_X, ZT_Z, IMM>;
      using Zp = ZTShape<NTR, ZT_X, ZT_Z, false>;
      R *t = static_cast<R *>(txy);
      const int nch = int(blocks(cfg.nz, ZT_Z));
      const int ci0 = !IMM ? 0 : (cfg.bc_z == PU_BC_WALL ? std::min(nch, (imm_levels() + 5 + ZT_Z - 1) / ZT_Z) : nch);
      const int ci = std::min(std::max(ci0, c0), c1);
      const bool tma = zt_tma && static_cast<const void *>(sin) == s[b];
      const unsigned bx = blocks(cfg.nx, ZT_X), by = unsigned(cfg.ny);
      if (ci > c0) {
        Grid<R> Gi = G;
        Gi.c_first = c0;
        const dim3 gt(bx, by, ci - c0);
        if (tma)
          k_zt<NTR, ZT_X, ZT_Z, IMM, true><<<gt, ZT_X * ZT_Z, Zs::tma_bytes, st>>>(Gi, sin, sn, sout, t, a_n, a_dt,
                                                                                 n_enforce, zt_maps[b]);
        else
          k_zt<NTR, ZT_X, ZT_Z, IMM><<<gt, ZT_X * ZT_Z, Zs::bytes, st>>>(Gi, sin, sn, sout, t, a_n, a_dt, n_enforce,
                                                                          zt_maps[b]);
        PU_LAUNCHED();
      }
      if (ci < c1) {
        Grid<R> Gp = G;
        Gp.c_first = ci;
        const dim3 gt(bx, by, c1 - ci);
        if (tma)
          k_zt<NTR, ZT_X, ZT_Z, false, true><<<gt, ZT_X * ZT_Z, Zp::tma_bytes, st>>>(Gp, sin, sn, sout, t, a_n, a_dt,
                                                                                    n_enforce, zt_maps[b]);
        else
          k_zt<NTR, ZT_X, ZT_Z, false><<<gt, ZT_X * ZT_Z, Zp::bytes, st>>>(Gp, sin, sn, sout, t, a_n, a_dt,
                                                                            n_enforce, zt_maps[b]);
        PU_LAUNCHED();
      }
    }
    return PU_OK;
  }

  // One SSPRK3 stage: the x/y kernel (DEC: a decomposed tile reading its
  // received halo slabs), then the z march with the stage combination.
  template <bool IMM, bool LRN, bool DEC = false>
  int stage(const Grid<R> &G, const R *sin, const R *sn, R *sout, R a_n, R a_dt, int n_enforce) {
    constexpr bool L = LRN && std::is_same<R, float>::value && !DEC;
    R *t = static_cast<R *>(txy);
    cudaEvent_t e0 = prof_begin();
    int b = 0;   // sin is s[b]: the tensor maps of that buffer
    while (b < 2 && static_cast<const void *>(sin) != s[b]) b++;
    if (small_tile) {
      using Sh = XYShape<R, NTR, XTX_SM, XTY_SM, IMM, L>;
      dim3 g(blocks(cfg.nx, XTX_SM), blocks(cfg.ny, XTY_SM), cfg.nz);
      k_xy<R, NTR, XTX_SM, XTY_SM, IMM, L, DEC><<<g, Sh::NT, Sh::bytes, st>>>(G, sin, t, xy_maps[b]);
      PU_LAUNCHED();
    } else if (L) {
      using Sh = XYShape<R, NTR, LTX, LTY, IMM, L>;
      dim3 g(blocks(cfg.nx, LTX), blocks(cfg.ny, LTY), cfg.nz);
      k_xy<R, NTR, LTX, LTY, IMM, L><<<g, Sh::NT, Sh::bytes, st>>>(G, sin, t, xy_maps[b]);
      PU_LAUNCHED();
    } else if (DEC && dec_edges_only) {
      // The tiles around the interior ones, which ran while the halos crossed.
      int tx0, tx1, ty0, ty1;
      dec_interior(tx0, tx1, ty0, ty1);
      const int nbx = int(blocks(cfg.nx, XTX_BIG)), nby = int(blocks(cfg.ny, XTY_BIG));
      PU_TRY((xy_levels<IMM, DEC>(G, sin, b, 0, cfg.nz, 0, nbx, 0, ty0)));
      PU_TRY((xy_levels<IMM, DEC>(G, sin, b, 0, cfg.nz, 0, nbx, ty1, nby)));
      PU_TRY((xy_levels<IMM, DEC>(G, sin, b, 0, cfg.nz, 0, tx0, ty0, ty1)));
      PU_TRY((xy_levels<IMM, DEC>(G, sin, b, 0, cfg.nz, tx1, nbx, ty0, ty1)));
    } else {
      PU_TRY((xy_levels<IMM, DEC>(G, sin, b, 0, cfg.nz)));
    }
    prof_end(0, e0);
    const int kc = cfg.z_chunk > 0 ? cfg.z_chunk : (cfg.nz < 16 ? cfg.nz : 16);
    dim3 gz(blocks(cfg.nx, ZTX), blocks(cfg.ny, ZTY), blocks(cfg.nz, kc));
    cudaEvent_t e1 = prof_begin();
    if constexpr (std::is_same<R, float>::value) {
      if (z_tiled(L)) {
        // z chunks [0, ci) take the immersed kernel: chunk c reads levels
        // 32c-5 .. 32c+36, so it is plain once 32c-5 reaches the first level
        // no flag holds.  A periodic z wraps flagged levels into the top
        // chunk: every chunk stays immersed there.  The maps of this stage
        // input (s[b]); the cell maps of sn and txy are the same for every b.
        PU_TRY((zt_chunks<IMM>(G, sin, sn, sout, a_n, a_dt, n_enforce, b, 0, int(blocks(cfg.nz, ZT_Z)))));
        prof_end(1, e1);
        return PU_OK;
      }
    }
    // The learned z march needs full warps: every block's columns inside the domain.
    if (L && cfg.nx % ZTX == 0 && cfg.ny % ZTY == 0)
      k_z<R, NTR, ZTX, ZTY, IMM, L><<<gz, ZTX * ZTY, ZShape<R, NTR, ZTX, ZTY, L>::bytes, st>>>(
          G, sin, sn, sout, t, a_n, a_dt, n_enforce, kc);
    else
      k_z<R, NTR, ZTX, ZTY, IMM><<<gz, ZTX * ZTY, ZShape<R, NTR, ZTX, ZTY>::bytes, st>>>(G, sin, sn, sout, t, a_n,
                                                                                       a_dt, n_enforce, kc);
    PU_LAUNCHED();
    prof_end(1, e1);
    return PU_OK;
  }

  template <bool IMM, bool LRN>
  int advance_t(double dt, int nsteps) {
    NvtxRange range("pu:advance");
    const Grid<R> G = grid();
    R *s0 = static_cast<R *>(s[0]), *s1 = static_cast<R *>(s[1]), *s2 = static_cast<R *>(s[2]);
    cudaEvent_t e0 = prof_begin();
    k_enforce<R, NTR, IMM><<<blocks(N, 256), 256, 0, st>>>(G, s0, 0, N);
    PU_LAUNCHED();
    prof_end(2, e0);
    for (int n = 0; n < nsteps; n++) {
      // Shu-Osher SSPRK(3,3) (dynamics_rk.h:308-360): s1 = s0 + dt L(s0);
      // s2 = 3/4 s0 + 1/4 (s1 + dt L(s1)); s0 <- 1/3 s0 + 2/3 (s2 + dt L(s2)).
      PU_TRY((stage<IMM, LRN>(G, s0, nullptr, s1, R(0), R(dt), 1)));
      PU_TRY((stage<IMM, LRN>(G, s1, s0, s2, R(3. / 4.), R(1. / 4. * dt), 1)));
      PU_TRY((stage<IMM, LRN>(G, s2, s0, s0, R(1. / 3.), R(2. / 3. * dt), n == nsteps - 1 ? 1 : 2)));
    }
    return PU_OK;
  }

  int advance(double dt, int nsteps) override {
    if (nsteps <= 0) return PU_OK;
    if (dc.on) {
      if (!has_transport()) {
        set_error("the tiles of an in-process group advance with pu_dycore_group_advance");
        return PU_ERR_STATE;
      }
      PU_TRY(dec_enforce());
      const bool split = dec_split();
      for (int n = 0; n < nsteps; n++)
        for (int sg = 0; sg < 3; sg++) {
          PU_TRY(dec_pack(sg));
          if (!split) {
            PU_TRY(exchange(dc.state, true, !sim2d()));
            PU_TRY(dec_compute(sg, dt, n == nsteps - 1));
            continue;
          }
          PU_TRY(exchange(dc.state, true, !sim2d(), [&] { return dec_xy_interior(sg); }));
          dec_edges_only = true;
          const int rc = dec_compute(sg, dt, n == nsteps - 1);
          dec_edges_only = false;
          PU_TRY(rc);
        }
      return PU_OK;
    }
    if (learned_active()) return has_imm ? advance_t<true, true>(dt, nsteps) : advance_t<false, true>(dt, nsteps);
    return has_imm ? advance_t<true, false>(dt, nsteps) : advance_t<false, false>(dt, nsteps);
  }

  // ---- time_step with the host copies overlapped ----
  // On host coupler arrays the copies in and out move 2 x 8 S N bytes over the
  // host link, as long as several steps on large grids.  Here the call runs
  // as a wavefront over chunks of ZT_Z levels: the input crosses chunk by
  // chunk on a copy stream, and stage g (1 .. 3 nsteps; 0 = the chunk's
  // conversion and enforcement) runs on chunk c once stage g-1 has run on
  // chunks c-1, c and c+1 (the z stencils reach 5 levels into each
  // neighbour).  On the one compute stream the launches go in diagonals
  // w = g + c, each in increasing g: everything in diagonal w waits only for
  // input chunk w, so the stages of the chunks already there run while the
  // rest crosses; each chunk's final state is converted back and copied out
  // while the others finish.  Every write lands after the reads of the old
  // values it replaces: stage g writes the buffer stage g-3 wrote, whose
  // readers (stage g-2 on c-1..c+1, and for s0 stages g-2 and g-1 on c) sit in
  // earlier diagonals or earlier in this one; the x/y tendency of chunk c is
  // written and read by the two kernels of one (g, c), in stream order.
  // Every cell gets the kernels and inputs of load_state + advance +
  // store_state, so the results are the same bits.  FP32 with the tiled z
  // kernel, walls in z (a periodic z couples the top and bottom chunks), at
  // least two chunks; the config's serial_io turns it off.
  bool io_overlap(const pu_state_view *v) const {
    if constexpr (!std::is_same<R, float>::value) {
      return false;
    } else {
      return !cfg.serial_io && !dc.on && !profiling && !small_tile && z_tiled(false) && !learned_active() &&
             cfg.bc_z == PU_BC_WALL && cfg.nz >= 2 * ZT_Z && v->rho_d &&
             resolve_mem(v->mem, v->rho_d) == PU_MEM_HOST;
    }
  }

  int time_step(pu_state_view *v, double dt, int nsteps) override {
    if (nsteps <= 0 || !io_overlap(v)) return ImplBase::time_step(v, dt, nsteps);
    double *host[5 + NTR] = {v->rho_d, v->uvel, v->vvel, v->wvel, v->temp};
    for (int t = 0; t < NTR; t++) host[5 + t] = v->tracers[t];
    for (int a = 0; a < 5 + NTR; a++)
      if (!host[a]) {
        set_error("coupler view has a null array");
        return PU_ERR_INVALID;
      }
    if (!cs) PU_CK(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    const int nch = int(blocks(cfg.nz, ZT_Z));
    while (io_ev.size() < size_t(2 * nch + 1)) {
      cudaEvent_t e;
      PU_CK(cudaEventCreateWithFlags(&e, cudaEventDisableTiming));
      io_ev.push_back(e);
    }
    const int rc = has_imm ? time_step_io<true>(host, dt, nsteps, nch) : time_step_io<false>(host, dt, nsteps, nch);
    // No copy into or out of the caller's arrays outlives the call.
    const cudaError_t e = cudaStreamSynchronize(cs);
    if (rc) return rc;
    if (e != cudaSuccess) {
      set_error(std::string("copy stream: ") + cudaGetErrorString(e));
      return PU_ERR_CUDA;
    }
    return check_err();
  }

  template <bool IMM>
  int time_step_io(double *const *host, double dt, int nsteps, int nch) {
    NvtxRange range("pu:time_step_overlapped");
    const Grid<R> G = grid();
    R *sb[3] = {static_cast<R *>(s[0]), static_cast<R *>(s[1]), static_cast<R *>(s[2])};
    CouplerPtrs cp;
    CouplerOut co;
    cp.rho_d = co.rho_d = staging;
    cp.u = co.u = staging + N;
    cp.v = co.v = staging + 2 * N;
    cp.w = co.w = staging + 3 * N;
    cp.T = co.T = staging + 4 * N;
    for (int t = 0; t < 8; t++) cp.tr[t] = co.tr[t] = t < NTR ? staging + size_t(5 + t) * N : nullptr;
    cudaEvent_t *ein = io_ev.data(), *eout = ein + nch, start = ein[2 * nch];
    auto lev = [&](int c) { return std::min(cfg.nz, c * ZT_Z); };
    const int last = 3 * nsteps;
    // The copy stream starts after the work queued so far (the staging
    // buffer is free then).
    PU_CK(cudaEventRecord(start, st));
    PU_CK(cudaStreamWaitEvent(cs, start, 0));
    // Stage g on chunk c: g = 0 brings the chunk in; g = 3n+1, 3n+2, 3n+3 are
    // the stages of step n as advance_t runs them (Shu-Osher SSPRK(3,3),
    // dynamics_rk.h:308-360); the last one also converts the chunk back.
    auto run = [&](int g, int c) -> int {
      const size_t e0 = size_t(lev(c)) * NP, e1 = size_t(lev(c + 1)) * NP;
      const unsigned nb = blocks(e1 - e0, 256);
      if (g == 0) {
        for (int a = 0; a < 5 + NTR; a++)
          PU_CK(cudaMemcpyAsync(staging + size_t(a) * N + e0, host[a] + e0, (e1 - e0) * sizeof(double),
                                cudaMemcpyHostToDevice, cs));
        PU_CK(cudaEventRecord(ein[c], cs));
        PU_CK(cudaStreamWaitEvent(st, ein[c], 0));
        k_load_coupler<R, NTR><<<nb, 256, 0, st>>>(cp, thermo(), rho_off, rt_off, N, NP, sb[0], e0, e1);
        PU_LAUNCHED();
        k_enforce<R, NTR, IMM><<<nb, 256, 0, st>>>(G, sb[0], e0, e1);
        PU_LAUNCHED();
        return PU_OK;
      }
      const int m = (g - 1) % 3;   // 0: s1 = s0 + dt L(s0); 1: s2 from s1; 2: s0 from s2
      const R a_n = m == 0 ? R(0) : (m == 1 ? R(3. / 4.) : R(1. / 3.));
      const R a_dt = m == 0 ? R(dt) : (m == 1 ? R(1. / 4. * dt) : R(2. / 3. * dt));
      const int n_enforce = (m == 2 && g != last) ? 2 : 1;
      PU_TRY((xy_levels<IMM>(G, sb[m], m, lev(c), lev(c + 1))));
      PU_TRY((zt_chunks<IMM>(G, sb[m], m == 0 ? nullptr : sb[0], sb[(m + 1) % 3], a_n, a_dt, n_enforce, m, c,
                             c + 1)));
      if (g == last) {
        k_store_coupler<R, NTR><<<nb, 256, 0, st>>>(co, thermo(), rho_off, rt_off, N, NP, sb[0], e0, e1);
        PU_LAUNCHED();
        PU_CK(cudaEventRecord(eout[c], st));
      }
      return PU_OK;
    };
    for (int w = 0; w <= last + nch - 1; w++)
      for (int g = std::max(0, w - (nch - 1)); g <= std::min(w, last); g++) PU_TRY(run(g, w - g));
    // The output copies, queued after all the compute so that a pageable
    // destination (whose copies hold the host thread) does not hold back the
    // launches.
    for (int c = 0; c < nch; c++) {
      const size_t e0 = size_t(lev(c)) * NP, e1 = size_t(lev(c + 1)) * NP;
      PU_CK(cudaStreamWaitEvent(cs, eout[c], 0));
      for (int a = 0; a < 5 + NTR; a++)
        PU_CK(cudaMemcpyAsync(host[a] + e0, staging + size_t(a) * N + e0, (e1 - e0) * sizeof(double),
                              cudaMemcpyDeviceToHost, cs));
    }
    return PU_OK;
  }

  // ---- decomposed tiles ----
  template <class T>
  int box(const T *src, int sxn, int syn, int si0, int sj0, T *dst, int dxn, int dyn, int di0, int dj0, int bx,
          int by, int bz) {
    const size_t n = size_t(bx) * by * bz;
    if (!n) return PU_OK;
    const unsigned nb = unsigned(std::min<size_t>((n + 255) / 256, size_t(148) * 16));
    k_box<T><<<nb, 256, 0, st>>>(src, sxn, syn, si0, sj0, dst, dxn, dyn, di0, dj0, bx, by, bz);
    PU_LAUNCHED();
    return PU_OK;
  }

  int dec_alloc() override {
    const size_t W = HALO_W, nz = cfg.nz, nx = cfg.nx, ny = cfg.ny;
    for (int d = 0; d < (sim2d() ? 2 : 4); d++) {
      const size_t b = size_t(S) * nz * (d < 2 ? ny * W : W * nx) * sizeof(R);
      unsigned char *p, *q;
      PU_TRY(dalloc(p, b));
      dc.state.snd[d] = p;
      PU_TRY(dalloc(q, b));
      dc.state.rcv[d] = q;
      dc.state.bytes[d] = b;
    }
    return PU_OK;
  }

  // The HALO_W columns (rows) of the stage input next to each x (y) edge.
  int dec_pack(int sg) override {
    const R *sin = static_cast<const R *>(s[sg]);
    const int nx = cfg.nx, ny = cfg.ny, W = HALO_W, P = S * cfg.nz;
    R **snd = reinterpret_cast<R **>(dc.state.snd);
    PU_TRY(box(sin, nx, ny, 0, 0, snd[0], W, ny, 0, 0, W, ny, P));
    PU_TRY(box(sin, nx, ny, nx - W, 0, snd[1], W, ny, 0, 0, W, ny, P));
    if (!sim2d()) {
      PU_TRY(box(sin, nx, ny, 0, 0, snd[2], nx, W, 0, 0, nx, W, P));
      PU_TRY(box(sin, nx, ny, 0, ny - W, snd[3], nx, W, 0, 0, nx, W, P));
    }
    return PU_OK;
  }

  int dec_enforce() override {
    const Grid<R> G = grid();
    R *s0 = static_cast<R *>(s[0]);
    if (has_imm) k_enforce<R, NTR, true><<<blocks(N, 256), 256, 0, st>>>(G, s0, 0, N);
    else k_enforce<R, NTR, false><<<blocks(N, 256), 256, 0, st>>>(G, s0, 0, N);
    PU_LAUNCHED();
    return PU_OK;
  }

  // Stage sg of the Shu-Osher SSPRK(3,3) step, as advance_t runs it.
  template <bool IMM>
  int dec_stage(const Grid<R> &G, int sg, double dt, bool last) {
    R *s0 = static_cast<R *>(s[0]), *s1 = static_cast<R *>(s[1]), *s2 = static_cast<R *>(s[2]);
    if (sg == 0) return stage<IMM, false, true>(G, s0, nullptr, s1, R(0), R(dt), 1);
    if (sg == 1) return stage<IMM, false, true>(G, s1, s0, s2, R(3. / 4.), R(1. / 4. * dt), 1);
    return stage<IMM, false, true>(G, s2, s0, s0, R(1. / 3.), R(2. / 3. * dt), last ? 1 : 2);
  }
  // The tiles of a decomposed tile's x/y kernel whose cross (the 16x16 tile
  // and 5 cells around it) stays inside the tile and so reads no halo slab:
  // [tx0, tx1) x [ty0, ty1), empty when the tile is too small.
  void dec_interior(int &tx0, int &tx1, int &ty0, int &ty1) const {
    tx0 = 1;
    ty0 = 1;
    tx1 = std::max(tx0, (cfg.nx - XTX_BIG - 5) / XTX_BIG + 1);
    ty1 = std::max(ty0, (cfg.ny - XTY_BIG - 5) / XTY_BIG + 1);
    if (cfg.nx < XTX_BIG + 5) tx1 = tx0;
    if (cfg.ny < XTY_BIG + 5) ty1 = ty0;
  }
  // Interior tiles run while the halos cross (a transport, the 16x16 x/y
  // tiles, some interior; the config's serial_io turns it off).
  bool dec_split() const {
    if (!dc.on || cfg.serial_io || small_tile || sim2d() || !has_transport()) return false;
    int tx0, tx1, ty0, ty1;
    dec_interior(tx0, tx1, ty0, ty1);
    return tx1 > tx0 && ty1 > ty0;
  }
  // The x/y kernel of stage sg on the interior tiles (the stage input is
  // s[sg]: s0, s1, s2 for the three stages).
  int dec_xy_interior(int sg) {
    const Grid<R> G = grid();
    const R *sin = static_cast<const R *>(s[sg]);
    int tx0, tx1, ty0, ty1;
    dec_interior(tx0, tx1, ty0, ty1);
    return has_imm ? xy_levels<true, true>(G, sin, sg, 0, cfg.nz, tx0, tx1, ty0, ty1)
                   : xy_levels<false, true>(G, sin, sg, 0, cfg.nz, tx0, tx1, ty0, ty1);
  }
  int dec_compute(int sg, double dt, bool last) override {
    const Grid<R> G = grid();
    return has_imm ? dec_stage<true>(G, sg, dt, last) : dec_stage<false>(G, sg, dt, last);
  }

  // Init of a tile, in phases between which the tiles exchange:
  //   begin: column sums of the tile; the immersed proportion (zeros for
  //          none, plus the windmill projection) and its INIT_HALO columns
  //          next to each x edge;
  //   (sum the column sums over the tiles)  hydro: the profiles;
  //   (x exchange)  mid: the x-extended proportion and its rows next to
  //          each y edge;
  //   (y exchange)  end: the extended block, immersed flags and relaxation
  //          factors on it, cropped to the tile and its halo slabs; the state.
  int dinit_begin(const pu_state_view *v, const double *prop, const double *proj, int mem) override {
    if (proj && !prop) {
      set_error("windmill_proj_weight needs immersed_proportion");
      return PU_ERR_INVALID;
    }
    CouplerPtrs cp;
    PU_TRY(device_view(v, cp));
    k_column_sums<NTR><<<cfg.nz, 256, 0, st>>>(cp, thermo(), cfg.nx, cfg.ny, sums);
    PU_LAUNCHED();
    PU_TRY(dalloc(dc.dprop, N));
    if (prop) {
      PU_CK(cudaMemcpyAsync(dc.dprop, prop, N * sizeof(double),
                            resolve_mem(mem, prop) == PU_MEM_DEVICE ? cudaMemcpyDeviceToDevice
                                                                    : cudaMemcpyHostToDevice,
                            st));
    } else {
      PU_CK(cudaMemsetAsync(dc.dprop, 0, N * sizeof(double), st));
    }
    if (proj) {
      double *dproj = nullptr;
      PU_TRY(dalloc(dproj, N));
      cudaMemcpyAsync(dproj, proj, N * sizeof(double),
                      resolve_mem(mem, proj) == PU_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, st);
      k_add_inplace<double><<<blocks(N, 256), 256, 0, st>>>(dc.dprop, dproj, N);
      const cudaError_t e = cudaGetLastError();
      cudaStreamSynchronize(st);
      cudaFree(dproj);
      if (e != cudaSuccess) {
        set_error(std::string("kernel launch: ") + cudaGetErrorString(e));
        return PU_ERR_CUDA;
      }
      launches++;
    }
    const int E = INIT_HALO, nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
    for (int d = 0; d < 2; d++) {
      const size_t b = size_t(nz) * ny * E * sizeof(double);
      unsigned char *p, *q;
      PU_TRY(dalloc(p, b));
      dc.ix.snd[d] = p;
      PU_TRY(dalloc(q, b));
      dc.ix.rcv[d] = q;
      dc.ix.bytes[d] = b;
    }
    double **snd = reinterpret_cast<double **>(dc.ix.snd);
    PU_TRY(box<double>(dc.dprop, nx, ny, 0, 0, snd[0], E, ny, 0, 0, E, ny, nz));
    PU_TRY(box<double>(dc.dprop, nx, ny, nx - E, 0, snd[1], E, ny, 0, 0, E, ny, nz));
    return PU_OK;
  }

  int dinit_hydro(const double *global_sums) override {
    if (global_sums) {
      PU_CK(cudaMemcpyAsync(sums, global_sums, size_t(3) * cfg.nz * sizeof(double), cudaMemcpyHostToDevice, st));
      PU_CK(cudaStreamSynchronize(st));
    }
    HydroOut ho{cells, edges, rho_off, rt_off};
    const double r = 1. / (double(dc.d.nx_glob) * double(dc.d.ny_glob));
    k_hydro_finish<R><<<1, HYDRO_THREADS, 0, st>>>(sums, cfg.nz, r, cfg.gamma_d, cfg.C0, cfg.grav, cfg.dz, sizeof(R) == 4, ho,
                                       lt);
    PU_LAUNCHED();
    return PU_OK;
  }

  int dinit_mid() override {
    const int E = INIT_HALO, nx = cfg.nx, ny = cfg.ny, nz = cfg.nz, nxe = nx + 2 * E;
    PU_TRY(dalloc(dc.ext_x, size_t(nz) * ny * nxe));
    const double *const *rcv = reinterpret_cast<double *const *>(dc.ix.rcv);
    PU_TRY(box<double>(dc.dprop, nx, ny, 0, 0, dc.ext_x, nxe, ny, E, 0, nx, ny, nz));
    PU_TRY(box<double>(rcv[0], E, ny, 0, 0, dc.ext_x, nxe, ny, 0, 0, E, ny, nz));
    PU_TRY(box<double>(rcv[1], E, ny, 0, 0, dc.ext_x, nxe, ny, E + nx, 0, E, ny, nz));
    if (sim2d()) return PU_OK;
    for (int d = 2; d < 4; d++) {
      const size_t b = size_t(nz) * E * nxe * sizeof(double);
      unsigned char *p, *q;
      PU_TRY(dalloc(p, b));
      dc.iy.snd[d] = p;
      PU_TRY(dalloc(q, b));
      dc.iy.rcv[d] = q;
      dc.iy.bytes[d] = b;
    }
    double **snd = reinterpret_cast<double **>(dc.iy.snd);
    PU_TRY(box<double>(dc.ext_x, nxe, ny, 0, 0, snd[2], nxe, E, 0, 0, nxe, E, nz));
    PU_TRY(box<double>(dc.ext_x, nxe, ny, 0, ny - E, snd[3], nxe, E, 0, 0, nxe, E, nz));
    return PU_OK;
  }

  int dinit_end(const pu_state_view *v) override {
    const int E = INIT_HALO, W = HALO_W, nx = cfg.nx, ny = cfg.ny, nz = cfg.nz;
    const int Ey = sim2d() ? 0 : E, nxe = nx + 2 * E, nye = ny + 2 * Ey;
    const size_t Ne = size_t(nz) * nye * nxe;
    const double *ext = dc.ext_x;
    if (!sim2d()) {
      PU_TRY(dalloc(dc.ext, Ne));
      const double *const *rcv = reinterpret_cast<double *const *>(dc.iy.rcv);
      PU_TRY(box<double>(dc.ext_x, nxe, ny, 0, 0, dc.ext, nxe, nye, 0, E, nxe, ny, nz));
      PU_TRY(box<double>(rcv[2], nxe, E, 0, 0, dc.ext, nxe, nye, 0, 0, nxe, E, nz));
      PU_TRY(box<double>(rcv[3], nxe, E, 0, 0, dc.ext, nxe, nye, 0, E + ny, nxe, E, nz));
      ext = dc.ext;
    }
    // Flags and factors of the extended block (the distance passes wrap in x
    // and y over the block; the wrap spans more than 10 cells from any cell
    // whose flags are kept, so it finds nothing).
    uint8_t *a = nullptr, *b = nullptr, *dz = nullptr, *fe = nullptr;
    R *me = nullptr;
    int rc = dalloc(a, Ne);
    if (!rc) rc = dalloc(b, Ne);
    if (!rc) rc = dalloc(dz, Ne);
    if (!rc) rc = dalloc(fe, Ne);
    if (!rc) rc = dalloc(me, Ne);
    if (!rc && !flags) rc = dalloc(flags, N);
    if (!rc && !imm_mult) {
      R *m;
      rc = dalloc(m, N);
      if (!rc) imm_mult = m;
    }
    for (int d = 0; d < (sim2d() ? 2 : 4) && !rc; d++)
      if (!dc.fslab[d]) rc = dalloc(dc.fslab[d], size_t(nz) * W * (d < 2 ? ny : nx));
    if (!rc) {
      k_dist_init<<<blocks(Ne, 256), 256, 0, st>>>(ext, 0, Ne, a, 10);
      for (int axis = 0; axis < 3; axis++) {
        k_dist_pass<<<blocks(Ne, 256), 256, 0, st>>>(a, b, nxe, nye, nz, axis, 10);
        std::swap(a, b);
      }
      k_dist_init<<<blocks(Ne, 256), 256, 0, st>>>(ext, 1, Ne, dz, 3);
      for (int axis = 0; axis < 3; axis++) {
        k_dist_pass<<<blocks(Ne, 256), 256, 0, st>>>(dz, b, nxe, nye, nz, axis, 3);
        cudaMemcpyAsync(dz, b, Ne, cudaMemcpyDeviceToDevice, st);
      }
      k_imm_finish<R><<<blocks(Ne, 256), 256, 0, st>>>(ext, a, dz, cfg.immersed_power, Ne, fe, me);
      const cudaError_t e = cudaGetLastError();
      if (e != cudaSuccess) {
        set_error(std::string("kernel launch: ") + cudaGetErrorString(e));
        rc = PU_ERR_CUDA;
      } else {
        launches += 9;
      }
    }
    if (!rc) rc = box<uint8_t>(fe, nxe, nye, E, Ey, flags, nx, ny, 0, 0, nx, ny, nz);
    if (!rc) rc = box<R>(me, nxe, nye, E, Ey, static_cast<R *>(imm_mult), nx, ny, 0, 0, nx, ny, nz);
    if (!rc) rc = box<uint8_t>(fe, nxe, nye, E - W, Ey, dc.fslab[0], W, ny, 0, 0, W, ny, nz);
    if (!rc) rc = box<uint8_t>(fe, nxe, nye, E + nx, Ey, dc.fslab[1], W, ny, 0, 0, W, ny, nz);
    if (!rc && !sim2d()) rc = box<uint8_t>(fe, nxe, nye, E, Ey - W, dc.fslab[2], nx, W, 0, 0, nx, W, nz);
    if (!rc && !sim2d()) rc = box<uint8_t>(fe, nxe, nye, E, Ey + ny, dc.fslab[3], nx, W, 0, 0, nx, W, nz);
    // The tile needs the immersed kernels if any of its cells has a flag
    // (immersed, or immersed cells within 10, its own or its neighbours') or
    // a halo cell is immersed.
    if (!rc) {
      std::vector<uint8_t> hf(N);
      cudaMemcpyAsync(hf.data(), flags, N, cudaMemcpyDeviceToHost, st);
      std::vector<uint8_t> hs[4];
      for (int d = 0; d < (sim2d() ? 2 : 4); d++) {
        hs[d].resize(size_t(nz) * W * (d < 2 ? ny : nx));
        cudaMemcpyAsync(hs[d].data(), dc.fslab[d], hs[d].size(), cudaMemcpyDeviceToHost, st);
      }
      const cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) {
        set_error(cudaGetErrorString(e));
        rc = PU_ERR_CUDA;
      }
      has_imm = false;
      for (size_t q = 0; q < N && !has_imm; q++) has_imm = hf[q] != 0;
      for (auto &h : hs)
        for (size_t q = 0; q < h.size() && !has_imm; q++) has_imm = (h[q] & FLAG_IMM) != 0;
    }
    cudaStreamSynchronize(st);
    for (void *p : {(void *)a, (void *)b, (void *)dz, (void *)fe, (void *)me})
      if (p) cudaFree(p);
    for (double **p : {&dc.dprop, &dc.ext_x, &dc.ext}) {
      if (*p) cudaFree(*p);
      *p = nullptr;
    }
    dc.ix.release();
    dc.iy.release();
    if (rc) return rc;
    PU_TRY(load_state(v));
    PU_CK(cudaStreamSynchronize(st));
    inited = true;
    return PU_OK;
  }

  int get_conserved(double *stp, double *trp, int mem) override {
    double *dst = staging;
    k_get_conserved<R, NTR><<<blocks(N, 256), 256, 0, st>>>(static_cast<const R *>(s[0]), rho_off, rt_off, N, NP,
                                                            dst, dst + 5 * N);
    PU_LAUNCHED();
    auto kind = resolve_mem(mem, stp) == PU_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost;
    PU_CK(cudaMemcpyAsync(stp, dst, 5 * N * sizeof(double), kind, st));
    if (trp) PU_CK(cudaMemcpyAsync(trp, dst + 5 * N, size_t(NTR) * N * sizeof(double), kind, st));
    PU_CK(cudaStreamSynchronize(st));
    return PU_OK;
  }

  int set_conserved(const double *stp, const double *trp, int mem) override {
    auto kind = resolve_mem(mem, stp) == PU_MEM_DEVICE ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice;
    PU_CK(cudaMemcpyAsync(staging, stp, 5 * N * sizeof(double), kind, st));
    PU_CK(cudaMemcpyAsync(staging + 5 * N, trp, size_t(NTR) * N * sizeof(double), kind, st));
    k_set_conserved<R, NTR><<<blocks(N, 256), 256, 0, st>>>(static_cast<R *>(s[0]), rho_off, rt_off, N, NP, staging,
                                                            staging + 5 * N);
    PU_LAUNCHED();
    PU_CK(cudaStreamSynchronize(st));
    return PU_OK;
  }

  int set_hydrostasis(const double *r, const double *t, const double *p) override {
    double *old_r = nullptr, *old_rt = nullptr;
    PU_TRY(dalloc(old_r, cfg.nz));
    int rc = dalloc(old_rt, cfg.nz);
    if (rc == PU_OK) {
      cudaMemcpyAsync(old_r, rho_off, cfg.nz * sizeof(double), cudaMemcpyDeviceToDevice, st);
      cudaMemcpyAsync(old_rt, rt_off, cfg.nz * sizeof(double), cudaMemcpyDeviceToDevice, st);
      std::vector<double> h(3 * size_t(nzh));
      for (int k = 0; k < nzh; k++) {
        double a = r[k], b = t[k], c = p[k];
        if (sizeof(R) == 4) { a = double(float(a)); b = double(float(b)); c = double(float(c)); }
        h[k] = a;
        h[nzh + k] = b;
        h[2 * nzh + k] = c;
      }
      cudaMemcpyAsync(cells, h.data(), h.size() * sizeof(double), cudaMemcpyHostToDevice, st);
      HydroOut ho{cells, edges, rho_off, rt_off};
      k_hydro_finish<R><<<1, HYDRO_THREADS, 0, st>>>(nullptr, cfg.nz, 0., cfg.gamma_d, cfg.C0, cfg.grav, cfg.dz, sizeof(R) == 4, ho,
                                         lt);
      launches++;
      k_rebase<R><<<blocks(N, 256), 256, 0, st>>>(static_cast<R *>(s[0]), old_r, old_rt, rho_off, rt_off, N, NP);
      launches++;
      cudaError_t e = cudaStreamSynchronize(st);
      if (e != cudaSuccess) { set_error(cudaGetErrorString(e)); rc = PU_ERR_CUDA; }
    }
    cudaFree(old_r);
    if (old_rt) cudaFree(old_rt);
    return rc;
  }

  int ml_harvest(long n, unsigned long long seed) override {
    int rc = ml_alloc();
    if (rc) return rc;
    rc = ml_reserve(ml_n + n);
    if (rc) return rc;
    const Grid<R> G = grid();
    k_harvest<R, NTR><<<blocks(size_t(n), 128), 128, 0, st>>>(G, static_cast<const R *>(s[0]), n, seed, ml_n,
                                                              ml_xs + size_t(ml_n) * 9, ml_ts + size_t(ml_n) * 5);
    PU_LAUNCHED();
    PU_CK(cudaStreamSynchronize(st));
    ml_n += n;
    return PU_OK;
  }

  // density_pert, theta_pert, pressure_pert of the coupler arrays against the
  // handle's cell profiles (the dycore's output hook).  Host outputs go
  // through the stage buffer s[1] (idle between steps; S*N values of R hold
  // 3*N doubles since S*sizeof(R) >= 24).
  int perturbations(const pu_state_view *v, double *dens, double *theta, double *press, int mem) override {
    CouplerPtrs cp;
    PU_TRY(device_view(v, cp));
    const bool dev = resolve_mem(mem, dens) == PU_MEM_DEVICE;
    double *out = static_cast<double *>(s[1]);
    k_perturbations<NTR><<<blocks(N, 256), 256, 0, st>>>(cp, thermo(), cells, nzh, N, NP, out);
    PU_LAUNCHED();
    double *dst[3] = {dens, theta, press};
    for (int a = 0; a < 3; a++)
      PU_CK(cudaMemcpyAsync(dst[a], out + size_t(a) * N, N * sizeof(double),
                            dev ? cudaMemcpyDeviceToDevice : cudaMemcpyDeviceToHost, st));
    PU_CK(cudaStreamSynchronize(st));
    return PU_OK;
  }

  int diagnostics(pu_diag *out) override {
    const double dV = cfg.dx * cfg.dy * cfg.dz;
    k_diag_partial<R, NTR><<<diag_blocks, 256, 0, st>>>(static_cast<const R *>(s[0]), rho_off, rt_off, N, NP, dV, cfg.dz,
                                                        cfg.grav, cfg.C0, cfg.gamma_d, diag_part);
    PU_LAUNCHED();
    k_diag_final<<<1, 32, 0, st>>>(diag_part, diag_blocks, 6 + NTR, diag_out);
    PU_LAUNCHED();
    double h[NDIAG] = {0};
    PU_CK(cudaMemcpyAsync(h, diag_out, (6 + NTR) * sizeof(double), cudaMemcpyDeviceToHost, st));
    PU_CK(cudaStreamSynchronize(st));
    out->mass = h[0];
    out->rho_theta = h[1];
    out->kinetic = h[2];
    out->internal = h[3];
    out->potential = h[4];
    out->total_energy = h[5];
    for (int t = 0; t < PU_MAX_TRACERS; t++) out->tracer_mass[t] = t < NTR ? h[6 + t] : 0.0;
    return PU_OK;
  }

  // Bytes of working memory a time step needs when every buffer is carved
  // out of one caller-provided region (each piece 256-byte aligned).
  static size_t scratch_bytes(const pu_config &c) {
    const size_t N = size_t(c.nx) * c.ny * c.nz, nzh = size_t(c.nz) + 2 * HS;
    auto al = [](size_t b) { return (b + 255) / 256 * 256; };
    return al(sizeof(int)) + al(3 * nzh * sizeof(double)) + al(3 * size_t(c.nz + 1) * sizeof(double)) +
           2 * al(size_t(c.nz) * sizeof(double)) +
           al((5 * nzh + 2 * size_t(c.nz + 1) + size_t(c.nz)) * sizeof(R)) + 4 * al(size_t(5 + NTR) * N * sizeof(R));
  }

  // time_step (dynamics_rk.h:103-137) on a device-resident coupler view with
  // the caller's hydrostatic cell profiles, every buffer taken from `scratch`
  // (no allocation).  The handle object lives on the stack and does not own
  // the buffers.
  static int noalloc_time_step(const pu_config &c, unsigned char *scratch, const double *dens_cells,
                               const double *theta_cells, const double *pressure_cells, pu_state_view *v,
                               double dt_phys, int *ncycles) {
    Impl im;
    im.owns = false;
    im.cfg = c;
    im.st = static_cast<cudaStream_t>(c.stream);
    im.ntr = NTR;
    im.F = 6 + NTR;
    im.S = 5 + NTR;
    im.N = size_t(c.nx) * c.ny * c.nz;
    im.NP = size_t(c.nx) * c.ny;
    im.nzh = c.nz + 2 * HS;
    unsigned char *p = scratch;
    auto take = [&](size_t b) {
      unsigned char *q = p;
      p += (b + 255) / 256 * 256;
      return q;
    };
    im.err = reinterpret_cast<int *>(take(sizeof(int)));
    im.cells = reinterpret_cast<double *>(take(3 * size_t(im.nzh) * sizeof(double)));
    im.edges = reinterpret_cast<double *>(take(3 * size_t(c.nz + 1) * sizeof(double)));
    im.rho_off = reinterpret_cast<double *>(take(size_t(c.nz) * sizeof(double)));
    im.rt_off = reinterpret_cast<double *>(take(size_t(c.nz) * sizeof(double)));
    R *tb = reinterpret_cast<R *>(take((5 * size_t(im.nzh) + 2 * size_t(c.nz + 1) + size_t(c.nz)) * sizeof(R)));
    im.lt.rho_h = tb;
    im.lt.theta_h = tb + im.nzh;
    im.lt.rt_inv = tb + 2 * im.nzh;
    im.lt.p0_h = tb + 3 * im.nzh;
    im.lt.dp_h = tb + 4 * im.nzh;
    im.lt.rho_e = tb + 5 * im.nzh;
    im.lt.theta_e = im.lt.rho_e + (c.nz + 1);
    im.lt.rt_target = im.lt.theta_e + (c.nz + 1);
    for (int b = 0; b < 3; b++) im.s[b] = take(size_t(im.S) * im.N * sizeof(R));
    im.txy = take(size_t(im.S) * im.N * sizeof(R));
    im.make_maps();
    int rc = im.configure();
    if (rc) return rc;
    // The array keeps the previous call's contents: the error word must start at zero.
    PU_CK(cudaMemsetAsync(im.err, 0, sizeof(int), im.st));
    const size_t nzh = im.nzh;
    PU_CK(cudaMemcpyAsync(im.cells, dens_cells, nzh * sizeof(double), cudaMemcpyHostToDevice, im.st));
    PU_CK(cudaMemcpyAsync(im.cells + nzh, theta_cells, nzh * sizeof(double), cudaMemcpyHostToDevice, im.st));
    PU_CK(cudaMemcpyAsync(im.cells + 2 * nzh, pressure_cells, nzh * sizeof(double), cudaMemcpyHostToDevice, im.st));
    HydroOut ho{im.cells, im.edges, im.rho_off, im.rt_off};
    k_hydro_finish<R><<<1, HYDRO_THREADS, 0, im.st>>>(nullptr, c.nz, 0., c.gamma_d, c.C0, c.grav, c.dz, sizeof(R) == 4, ho, im.lt);
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
      set_error(std::string("kernel launch: ") + cudaGetErrorString(e));
      return PU_ERR_CUDA;
    }
    im.inited = true;
    const double dt0 = c.cfl * std::fmin(std::fmin(c.dx, c.dy), c.dz) / (350. + 100.);
    const int n = (int)std::ceil(dt_phys / dt0);
    rc = im.load_state(v);
    if (!rc) rc = im.advance(dt_phys / n, n);
    if (!rc) rc = im.store_state(v);
    if (ncycles) *ncycles = n;
    return rc;
  }
#undef PU_TRY
};

}  // namespace pu
