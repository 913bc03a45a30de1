// C entry points of libpu_dycore (declared in include/pu_dycore.h).
#include <cuda_runtime.h>
#include <dlfcn.h>

#include <cmath>
#include <cstring>
#include <memory>
#include <mutex>
#include <string>
#include <type_traits>
#include <vector>

#include "impl.cuh"
#include "tc_limiter.cuh"

namespace pu {

namespace {
thread_local std::string g_error;
}
// Records the message of a failed call and clears the runtime's last error,
// so that a failure the caller recovers from (an allocation that did not fit,
// say) is not reported again by the next launch check.  A sticky error stays
// with the context whatever is cleared here.
void set_error(const std::string &msg) {
  g_error = msg;
  cudaGetLastError();
}

NcclApi &nccl() {
  static NcclApi api;
  static std::once_flag once;
  std::call_once(once, [] {
    void *lib = dlopen("libnccl.so.2", RTLD_NOW | RTLD_LOCAL);
    if (!lib) {
      const char *e = dlerror();
      api.error = std::string("cannot load libnccl.so.2: ") + (e ? e : "unknown error");
      return;
    }
    bool ok = true;
    auto get = [&](auto &fn, const char *name) {
      fn = reinterpret_cast<std::remove_reference_t<decltype(fn)>>(dlsym(lib, name));
      if (!fn && ok) {
        ok = false;
        api.error = std::string("libnccl.so.2 has no ") + name;
      }
    };
    get(api.GetUniqueId, "ncclGetUniqueId");
    get(api.CommInitRank, "ncclCommInitRank");
    get(api.CommDestroy, "ncclCommDestroy");
    get(api.GroupStart, "ncclGroupStart");
    get(api.GroupEnd, "ncclGroupEnd");
    get(api.Send, "ncclSend");
    get(api.Recv, "ncclRecv");
    get(api.AllReduce, "ncclAllReduce");
    get(api.AllGather, "ncclAllGather");
    get(api.GetErrorString, "ncclGetErrorString");
    api.ok = ok;
  });
  return api;
}

#define PU_DECL(tag) ImplBase *make_impl_##tag();
PU_DECL(f32_1) PU_DECL(f32_2) PU_DECL(f32_3) PU_DECL(f32_4)
PU_DECL(f64_1) PU_DECL(f64_2) PU_DECL(f64_3) PU_DECL(f64_4)
#undef PU_DECL

static ImplBase *make_impl(int precision, int ntr) {
  if (precision == PU_F32) {
    switch (ntr) {
      case 1: return make_impl_f32_1();
      case 2: return make_impl_f32_2();
      case 3: return make_impl_f32_3();
      case 4: return make_impl_f32_4();
    }
  } else {
    switch (ntr) {
      case 1: return make_impl_f64_1();
      case 2: return make_impl_f64_2();
      case 3: return make_impl_f64_3();
      case 4: return make_impl_f64_4();
    }
  }
  return nullptr;
}

}  // namespace pu

using pu::set_error;

struct pu_dycore {
  std::unique_ptr<pu::ImplBase> impl;
  int device = 0;
};

namespace {

int fail(int code, const std::string &msg) {
  set_error(msg);
  return code;
}

// Every entry point runs with the handle's device current and restores the
// caller's device afterwards.
// Makes a handle's device current for one call and restores the caller's
// device afterwards; `status` is the switch's result (nothing may run on the
// device when it failed).
struct DeviceGuard {
  int prev = -1;
  cudaError_t status = cudaSuccess;
  explicit DeviceGuard(int dev) {
    if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
    if (prev != dev) status = cudaSetDevice(dev);
  }
  ~DeviceGuard() {
    int cur = -1;
    if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
  }
};

// Declares the guard of a call and returns PU_ERR_CUDA from it when the device
// cannot be made current.
#define PU_DEVICE_GUARD(dev)                                                                 \
  DeviceGuard g(dev);                                                                        \
  if (g.status != cudaSuccess)                                                               \
  return fail(PU_ERR_CUDA, std::string("cudaSetDevice: ") + cudaGetErrorString(g.status))

}  // namespace

namespace pu {
int check_config(const pu_config *c) {
  if (!c) return fail(PU_ERR_INVALID, "null config");
  if (c->nx < 1 || c->ny < 1 || c->nz < 1) return fail(PU_ERR_INVALID, "grid dimensions must be positive");
  if (c->nx < PU_HS + 1 && c->bc_x == PU_BC_PERIODIC)
    return fail(PU_ERR_UNSUPPORTED, "nx must exceed the halo width for periodic x");
  if (c->nz < PU_HS) return fail(PU_ERR_UNSUPPORTED, "nz must be at least the halo width");
  if (!(c->dx > 0 && c->dy > 0 && c->dz > 0)) return fail(PU_ERR_INVALID, "grid spacing must be positive");
  if (c->ntracers < 1 || c->ntracers > PU_MAX_TRACERS)
    return fail(PU_ERR_UNSUPPORTED, "the dycore needs 1..PU_MAX_TRACERS tracers (water_vapor is required)");
  if (c->idWV < 0 || c->idWV >= c->ntracers) return fail(PU_ERR_INVALID, "idWV must index the water_vapor tracer");
  if (c->bc_x != PU_BC_PERIODIC && c->bc_x != PU_BC_PRECURSOR) return fail(PU_ERR_INVALID, "bc_x must be periodic or precursor");
  if (c->bc_y != PU_BC_PERIODIC && c->bc_y != PU_BC_PRECURSOR) return fail(PU_ERR_INVALID, "bc_y must be periodic or precursor");
  if (c->bc_z != PU_BC_WALL && c->bc_z != PU_BC_PERIODIC)
    return fail(PU_ERR_INVALID, "ERROR: Specified invalid bc_z in coupler options");
  if (c->precision != PU_F32 && c->precision != PU_F64) return fail(PU_ERR_INVALID, "precision must be PU_F32 or PU_F64");
  if (c->weno_mode != PU_WENO_PLAIN && c->weno_mode != PU_WENO_LEARNED) return fail(PU_ERR_INVALID, "bad WENO mode");
  if (!(c->gamma_d > 1 && c->C0 > 0 && c->R_d > 0 && c->cfl > 0)) return fail(PU_ERR_INVALID, "bad thermodynamic options");
  if (c->z_chunk < 0) return fail(PU_ERR_INVALID, "z_chunk must be >= 0");
  if (c->thread_loads != 0 && c->thread_loads != 1) return fail(PU_ERR_INVALID, "thread_loads must be 0 or 1");
  if (c->imm_all_levels != 0 && c->imm_all_levels != 1) return fail(PU_ERR_INVALID, "imm_all_levels must be 0 or 1");
  if (c->serial_io != 0 && c->serial_io != 1) return fail(PU_ERR_INVALID, "serial_io must be 0 or 1");
  return PU_OK;
}
}  // namespace pu

namespace {
using pu::check_config;
}  // namespace

namespace {

// ---------------------------------------------------------------------------
// Decomposition geometry (coupler.h:132-229) and the tiles of a group.
// ---------------------------------------------------------------------------
// coupler.h:148-171, including its choice rule: each candidate nproc_y is
// compared through choice/(nranks/best-so-far), the first of equal distances
// wins, and ny_glob == 1 gives nranks x 1.
void process_grid(int nranks, long long nx_glob, long long ny_glob, int &npx, int &npy) {
  if (ny_glob == 1) {
    npx = nranks;
    npy = 1;
    return;
  }
  std::vector<double> choices;
  for (int q = 1; q <= nranks; q++)
    if (nranks % q == 0) choices.push_back(q);
  const double aspect_real = double(ny_glob) / double(nx_glob);
  npy = int(choices.at(0));
  double aspect = double(npy) / (nranks / npy);
  double min_dist = std::abs(aspect - aspect_real);
  for (size_t i = 1; i < choices.size(); i++) {
    aspect = choices[i] / (nranks / npy);
    const double dist = std::abs(aspect - aspect_real);
    if (dist < min_dist) {
      npy = int(choices[i]);
      min_dist = dist;
    }
  }
  npx = nranks / npy;
}

// coupler.h:176-183.
void tile_range(long long n_glob, int nproc, int p, long long &beg, long long &n) {
  const double nper = double(n_glob) / nproc;
  beg = (long long)std::round(nper * p);
  const long long end = (long long)(std::round(nper * (p + 1)) - 1);
  n = end - beg + 1;
}

void neighbors(const pu_decomp &d, int nbr[4]) {
  auto rank = [&](int px, int py) {
    px = ((px % d.nproc_x) + d.nproc_x) % d.nproc_x;
    py = ((py % d.nproc_y) + d.nproc_y) % d.nproc_y;
    return py * d.nproc_x + px;
  };
  nbr[0] = rank(d.px - 1, d.py);
  nbr[1] = rank(d.px + 1, d.py);
  nbr[2] = rank(d.px, d.py - 1);
  nbr[3] = rank(d.px, d.py + 1);
}

int check_decomp(const pu_decomp *d, const pu_config &c) {
  if (d->nproc_x < 1 || d->nproc_y < 1 || d->px < 0 || d->px >= d->nproc_x || d->py < 0 || d->py >= d->nproc_y)
    return fail(PU_ERR_INVALID, "bad tile grid or tile position");
  if (d->nx_glob < c.nx || d->ny_glob < c.ny) return fail(PU_ERR_INVALID, "the tile is larger than the global grid");
  if (d->ny_glob == 1) {
    if (d->nproc_y != 1 || c.ny != 1) return fail(PU_ERR_INVALID, "ny_glob == 1 needs one tile row with ny = 1");
  } else if (c.ny < pu::INIT_HALO) {
    return fail(PU_ERR_INVALID, "decomposed tiles need ny >= 12");
  }
  if (c.nx < pu::INIT_HALO) return fail(PU_ERR_INVALID, "decomposed tiles need nx >= 12");
  return PU_OK;
}

struct TileInfo {
  int px, py, nx, ny, nz, S, precision;
};

// Every tile of the grid once; tiles in a column of the grid (same px) of
// equal nx, in a row of equal ny, adding up to the global grid; nz, the
// field count and the precision equal.
bool tiles_fit(const pu_decomp &d, const std::vector<TileInfo> &t, std::string &why) {
  const int n = d.nproc_x * d.nproc_y;
  if (int(t.size()) != n) {
    why = "the group does not hold every tile of the grid";
    return false;
  }
  std::vector<const TileInfo *> at(n, nullptr);
  for (auto &x : t) {
    if (x.px < 0 || x.px >= d.nproc_x || x.py < 0 || x.py >= d.nproc_y) {
      why = "a tile lies outside the grid";
      return false;
    }
    const TileInfo *&slot = at[x.py * d.nproc_x + x.px];
    if (slot) {
      why = "two tiles share one grid position";
      return false;
    }
    slot = &x;
  }
  long long sx = 0, sy = 0;
  for (int py = 0; py < d.nproc_y; py++)
    for (int px = 0; px < d.nproc_x; px++) {
      const TileInfo &a = *at[py * d.nproc_x + px], &o = *at[0];
      if (a.nz != o.nz || a.S != o.S || a.precision != o.precision) {
        why = "tiles differ in nz, tracer count or precision";
        return false;
      }
      if (a.nx != at[px]->nx || a.ny != at[py * d.nproc_x]->ny) {
        why = "tiles of one grid column differ in nx, or of one grid row in ny";
        return false;
      }
      if (py == 0) sx += a.nx;
      if (px == 0) sy += a.ny;
    }
  if (sx != d.nx_glob || sy != d.ny_glob) {
    why = "the tile sizes do not add up to the global grid";
    return false;
  }
  return true;
}

int set_decomposition(pu::ImplBase &I, const pu_decomp &d, const unsigned char *id) {
  auto &dc = I.dc;
  dc.d = d;
  dc.rank = d.py * d.nproc_x + d.px;
  dc.nranks = d.nproc_x * d.nproc_y;
  neighbors(d, dc.nbr);
  int rc = I.dec_alloc();
  if (rc) return rc;
  if (id) {
    auto &api = pu::nccl();
    if (!api.ok) return fail(PU_ERR_UNSUPPORTED, api.error);
    ncclUniqueId u;
    std::memcpy(u.internal, id, sizeof(u.internal));
    ncclResult_t r = api.CommInitRank(&dc.comm, dc.nranks, u, dc.rank);
    if (r != ncclSuccess) {
      dc.comm = nullptr;
      return fail(PU_ERR_CUDA, std::string("ncclCommInitRank: ") + api.GetErrorString(r));
    }
    // Every rank checks the whole table of tiles, so a misfit fails on all
    // ranks alike before any halo is exchanged.
    const TileInfo mine{d.px, d.py, I.cfg.nx, I.cfg.ny, I.cfg.nz, I.S, I.cfg.precision};
    int *buf = nullptr;
    const size_t ni = sizeof(TileInfo) / sizeof(int);
    if (cudaMalloc(&buf, ni * (dc.nranks + 1) * sizeof(int)) != cudaSuccess) return fail(PU_ERR_NOMEM, "cudaMalloc");
    std::vector<TileInfo> all(dc.nranks);
    cudaMemcpyAsync(buf, &mine, sizeof(TileInfo), cudaMemcpyHostToDevice, I.st);
    r = api.AllGather(buf, buf + ni, ni, ncclInt32, dc.comm, I.st);
    cudaMemcpyAsync(all.data(), buf + ni, sizeof(TileInfo) * dc.nranks, cudaMemcpyDeviceToHost, I.st);
    const cudaError_t e = cudaStreamSynchronize(I.st);
    cudaFree(buf);
    if (r != ncclSuccess) return fail(PU_ERR_CUDA, std::string("ncclAllGather: ") + api.GetErrorString(r));
    if (e != cudaSuccess) return fail(PU_ERR_CUDA, cudaGetErrorString(e));
    std::string why;
    if (!tiles_fit(d, all, why)) return fail(PU_ERR_INVALID, why);
  }
  dc.on = true;
  return PU_OK;
}

// The tiles of an in-process group, indexed by rank; all checks first.
int group_tiles(pu_dycore *const *hs, int n, std::vector<pu::ImplBase *> &byrank, bool need_init) {
  if (!hs || n < 1) return fail(PU_ERR_INVALID, "empty group");
  for (int i = 0; i < n; i++)
    if (!hs[i] || !hs[i]->impl) return fail(PU_ERR_INVALID, "null handle in the group");
  const pu::ImplBase &h0 = *hs[0]->impl;
  std::vector<TileInfo> info;
  byrank.assign(n, nullptr);
  for (int i = 0; i < n; i++) {
    pu::ImplBase &I = *hs[i]->impl;
    if (!I.dc.on || I.dc.comm || I.dc.host)
      return fail(PU_ERR_STATE, "group tiles are made with pu_dycore_set_decomposition(h, d, NULL)");
    if (I.dc.d.nproc_x != h0.dc.d.nproc_x || I.dc.d.nproc_y != h0.dc.d.nproc_y ||
        I.dc.d.nx_glob != h0.dc.d.nx_glob || I.dc.d.ny_glob != h0.dc.d.ny_glob)
      return fail(PU_ERR_INVALID, "group tiles differ in their tile grid");
    if (hs[i]->device != hs[0]->device || I.st != h0.st)
      return fail(PU_ERR_INVALID, "group tiles must share one device and one stream");
    if (need_init && !I.inited) return fail(PU_ERR_STATE, "pu_dycore_group_init has not been called");
    if (I.dc.rank < 0 || I.dc.rank >= n || byrank[I.dc.rank]) return fail(PU_ERR_INVALID, "bad or repeated tile");
    byrank[I.dc.rank] = &I;
    info.push_back({I.dc.d.px, I.dc.d.py, I.cfg.nx, I.cfg.ny, I.cfg.nz, I.S, I.cfg.precision});
  }
  std::string why;
  if (!tiles_fit(h0.dc.d, info, why)) return fail(PU_ERR_INVALID, why);
  return PU_OK;
}

// Every tile's rcv[d] <- its neighbour's snd[d ^ 1] (one stream, in order).
int local_exchange(std::vector<pu::ImplBase *> &t, int which, bool x, bool y) {
  for (pu::ImplBase *a : t) {
    pu::HaloSet &ha = a->halo(which);
    for (int d = 0; d < 4; d++) {
      if ((d < 2 && !x) || (d >= 2 && !y)) continue;
      pu::HaloSet &hb = t[a->dc.nbr[d]]->halo(which);
      if (ha.bytes[d] != hb.bytes[d ^ 1]) return fail(PU_ERR_INVALID, "neighbouring tiles do not fit");
      if (cudaMemcpyAsync(ha.rcv[d], hb.snd[d ^ 1], ha.bytes[d], cudaMemcpyDeviceToDevice, a->st) != cudaSuccess)
        return fail(PU_ERR_CUDA, "halo copy failed");
    }
  }
  return PU_OK;
}

}  // namespace

namespace {

// The learned path's input normalisation (normalize9) on n stencils: x = the
// stencil scaled to [0,1] by its range, jump = the largest normalised
// neighbour difference (the acceptance check).
__global__ void k_normalize9_eval(const float *__restrict__ s, long long n, float *__restrict__ x,
                                  float *__restrict__ jump) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i >= n) return;
  float st[9], xs[9];
#pragma unroll
  for (int m = 0; m < 9; m++) st[m] = s[i * 9 + m];
  const float j = pu::normalize9(st, xs);
#pragma unroll
  for (int m = 0; m < 9; m++) x[i * 9 + m] = xs[m];
  jump[i] = j;
}

// A bounded wait that runs out: thread 0 announces 16 bytes of copies on an
// mbarrier of the block and issues none, so the barrier's phase never
// completes; every thread waits on it with the wait of the stage kernels' TMA
// staging (pu::tma::mbar_wait) for at most limit_ns and gives up.  out[0] = 1
// if any thread saw the phase complete (none can), out[1] = the clock cycles
// thread 0 waited.
__global__ void k_wait_check(unsigned long long limit_ns, long long *out) {
  __shared__ __align__(8) uint64_t bar;
  if (threadIdx.x == 0) {
    pu::tma::mbar_init(&bar);
    pu::tma::mbar_expect(&bar, 16u);
  }
  __syncthreads();
  const long long t0 = clock64();
  const bool ok = pu::tma::mbar_wait(&bar, 0, limit_ns);
  const long long t1 = clock64();
  const int any = __syncthreads_or(ok);
  if (threadIdx.x == 0) {
    out[0] = any;
    out[1] = t1 - t0;
  }
}

// The FP32 limiter on a batch of stencils: VARIANT 0 the scalar form, 1 the
// packed form (stencils 2i and 2i+1 in one thread), 4 the packed one-edge
// form (the right edge of stencil 2i and the left edge of stencil 2i+1; the
// other two outputs of the pair are NaN).
template <int VARIANT>
__global__ void k_weno9_eval(const float *__restrict__ s, const unsigned char *__restrict__ flags, long long n,
                             float *__restrict__ qL, float *__restrict__ qR) {
  const long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if constexpr (VARIANT == 0) {
    if (i >= n) return;
    float st[9];
#pragma unroll
    for (int m = 0; m < 9; m++) st[m] = s[i * 9 + m];
    const unsigned f = flags ? flags[i] : 1u;
    float a, b;
    pu::weno9_edges<float>(st, a, b, (f & 1u) != 0, (f & 2u) != 0, (f & 4u) != 0);
    qL[i] = a;
    qR[i] = b;
  } else {
    const long long a = 2 * i, b = 2 * i + 1;
    if (a >= n) return;
    const long long bb = b < n ? b : a;
    float2 st[9];
#pragma unroll
    for (int m = 0; m < 9; m++) st[m] = make_float2(s[a * 9 + m], s[bb * 9 + m]);
    const unsigned fa = flags ? flags[a] : 1u, fb = flags ? flags[bb] : 1u;
    const pu::bool2 mp{(fa & 1u) != 0, (fb & 1u) != 0}, il{(fa & 2u) != 0, (fb & 2u) != 0},
        ir{(fa & 4u) != 0, (fb & 4u) != 0};
    if constexpr (VARIANT == 1) {
      float2 L, R;
      pu::weno9_edges2(st, L, R, mp, il, ir);
      qL[a] = L.x;
      qR[a] = R.x;
      if (b < n) {
        qL[b] = L.y;
        qR[b] = R.y;
      }
    } else {
      const float2 q = pu::weno9_outer_edges2(st, mp, il, ir);
      qL[a] = __int_as_float(0x7fc00000);
      qR[a] = q.x;
      if (b < n) {
        qL[b] = q.y;
        qR[b] = __int_as_float(0x7fc00000);
      }
    }
  }
}

// The FP32 limiter with its linear forms on the tensor cores
// (tc_limiter.cuh): 128 stencils per block and round, one per thread.  The
// waits on the MMA are bounded; a round whose MMA did not complete sets *err
// and ends the kernel after releasing the tensor memory.
__global__ void __launch_bounds__(128) k_weno9_tc(const float *__restrict__ s, const unsigned char *__restrict__ flags,
                                                  long long n, float *__restrict__ qL, float *__restrict__ qR,
                                                  int *err) {
  namespace tc = pu::tc;
  __shared__ __align__(1024) uint32_t a_hi[tc::TC_A_WORDS], a_lo[tc::TC_A_WORDS];
  __shared__ __align__(1024) uint32_t b_hi[tc::TC_B_WORDS], b_lo[tc::TC_B_WORDS];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t taddr_s;
  const int tid = threadIdx.x, warp = tid >> 5;
  tc::fill_coefs(b_hi, b_lo);
  const uint32_t mb = tc::smem_addr(&mbar);
  if (tid == 0) tc::mbar_init(mb);
  if (warp == 0) tc::tmem_alloc(tc::smem_addr(&taddr_s), 32);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  uint32_t phase = 0;
  for (long long b0 = (long long)blockIdx.x * 128; b0 < n; b0 += (long long)gridDim.x * 128) {
    const long long i = b0 + tid;
    float st[9];
#pragma unroll
    for (int m = 0; m < 9; m++) st[m] = i < n ? s[i * 9 + m] : 0.f;
    tc::stage_row(st, tid, a_hi, a_lo);
    tc::fence_async_smem();
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      tc::issue(taddr, a_hi, a_lo, b_hi, b_lo);
      tc::commit(mb);
    }
    const bool ok = __syncthreads_and(tc::mbar_wait(mb, phase));
    phase ^= 1u;
    if (!ok) {
      if (tid == 0) atomicOr(err, 1);
      break;
    }
    tc::fence_after_sync();
    uint32_t r[32];
    tc::tmem_ld32(taddr + (uint32_t(warp * 32) << 16), r);
    if (i < n) {
      const unsigned f = flags ? flags[i] : 1u;
      float a, b;
      tc::edges_from_row(r, st[4], a, b, (f & 1u) != 0, (f & 2u) != 0, (f & 4u) != 0);
      qL[i] = a;
      qR[i] = b;
    }
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, 32);
}

// As k_weno9_tc with the A operand in tensor memory: 256 threads, two
// halves of 128 rows on the same 128 lanes, A of half h in columns
// 16h..16h+15 (hi, lo), its accumulator in columns 32+32h..; 128 columns.
__global__ void __launch_bounds__(256) k_weno9_tc_ts(const float *__restrict__ s,
                                                     const unsigned char *__restrict__ flags, long long n,
                                                     float *__restrict__ qL, float *__restrict__ qR, int *err) {
  namespace tc = pu::tc;
  __shared__ __align__(1024) uint32_t b_hi[tc::TC_B_WORDS], b_lo[tc::TC_B_WORDS];
  __shared__ __align__(8) unsigned long long mbar;
  __shared__ uint32_t taddr_s;
  const int tid = threadIdx.x, warp = tid >> 5, half = tid >> 7;
  tc::fill_coefs(b_hi, b_lo);
  const uint32_t mb = tc::smem_addr(&mbar);
  if (tid == 0) tc::mbar_init(mb);
  if (warp == 0) tc::tmem_alloc(tc::smem_addr(&taddr_s), 128);
  tc::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t taddr = taddr_s;
  const uint32_t lane_base = uint32_t((warp & 3) * 32) << 16;
  const uint64_t bh = tc::smem_desc(tc::smem_addr(b_hi)), bl = tc::smem_desc(tc::smem_addr(b_lo));
  uint32_t phase = 0;
  for (long long b0 = (long long)blockIdx.x * 256; b0 < n; b0 += (long long)gridDim.x * 256) {
    const long long i = b0 + tid;
    float st[9];
#pragma unroll
    for (int m = 0; m < 9; m++) st[m] = i < n ? s[i * 9 + m] : 0.f;
    uint32_t v[16];
    tc::split_row(st, v);
    tc::tmem_st16(taddr + lane_base + uint32_t(16 * half), v);
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
#pragma unroll
      for (int h = 0; h < 2; h++) {
        const uint32_t a = taddr + uint32_t(16 * h), d = taddr + uint32_t(32 + 32 * h);
        tc::mma_tf32_ts(d, a + 8, bh, 0u);
        tc::mma_tf32_ts(d, a, bl, 1u);
        tc::mma_tf32_ts(d, a, bh, 1u);
      }
      tc::commit(mb);
    }
    const bool ok = __syncthreads_and(tc::mbar_wait(mb, phase));
    phase ^= 1u;
    if (!ok) {
      if (tid == 0) atomicOr(err, 1);
      break;
    }
    tc::fence_after_sync();
    uint32_t r[32];
    tc::tmem_ld32(taddr + lane_base + uint32_t(32 + 32 * half), r);
    if (i < n) {
      const unsigned f = flags ? flags[i] : 1u;
      float a, b;
      tc::edges_from_row(r, st[4], a, b, (f & 1u) != 0, (f & 2u) != 0, (f & 4u) != 0);
      qL[i] = a;
      qR[i] = b;
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  tc::fence_before_sync();
  __syncthreads();
  if (warp == 0) tc::tmem_dealloc(taddr, 128);
}

}  // namespace

extern "C" {

int pu_version(void) { return 100; }

const char *pu_last_error(void) { return pu::g_error.c_str(); }

int pu_dycore_create(const pu_config *cfg, pu_dycore **out) {
  if (!out) return fail(PU_ERR_INVALID, "null output pointer");
  *out = nullptr;
  int rc = check_config(cfg);
  if (rc) return rc;
  int ndev = 0;
  if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return fail(PU_ERR_CUDA, "no CUDA device");
  if (cfg->device < 0 || cfg->device >= ndev) return fail(PU_ERR_INVALID, "bad device ordinal");
  PU_DEVICE_GUARD(cfg->device);
  std::unique_ptr<pu_dycore> h(new pu_dycore);
  h->device = cfg->device;
  h->impl.reset(pu::make_impl(cfg->precision, cfg->ntracers));
  if (!h->impl) return fail(PU_ERR_UNSUPPORTED, "no implementation for this precision/tracer count");
  auto &I = *h->impl;
  I.cfg = *cfg;
  I.st = static_cast<cudaStream_t>(cfg->stream);
  I.ntr = cfg->ntracers;
  I.N = size_t(cfg->nx) * cfg->ny * cfg->nz;
  I.NP = size_t(cfg->nx) * cfg->ny;
  I.nzh = cfg->nz + 2 * PU_HS;
  I.weno_mode = cfg->weno_mode;
  rc = I.alloc();
  if (rc) return rc;
  *out = h.release();
  return PU_OK;
}

int pu_dycore_destroy(pu_dycore *h) {
  if (!h) return PU_OK;
  {
    DeviceGuard g(h->device);
    if (h->impl) cudaStreamSynchronize(h->impl->st);
    h->impl.reset();
  }
  delete h;
  return PU_OK;
}

int pu_dycore_init(pu_dycore *h, const pu_state_view *coupler, const double *immersed_proportion, int mem) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  PU_DEVICE_GUARD(h->device);
  return h->impl->init(coupler, immersed_proportion, mem);
}

int pu_dycore_init_windmill(pu_dycore *h, const pu_state_view *coupler, const double *immersed_proportion,
                            const double *windmill_proj_weight, int mem) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (windmill_proj_weight && !immersed_proportion)
    return fail(PU_ERR_INVALID, "windmill_proj_weight needs immersed_proportion");
  PU_DEVICE_GUARD(h->device);
  return h->impl->init(coupler, immersed_proportion, mem, windmill_proj_weight);
}

int pu_dycore_compute_time_step(const pu_dycore *h, double *dt) {
  if (!h || !dt) return fail(PU_ERR_INVALID, "null argument");
  const pu_config &c = h->impl->cfg;
  const double maxwave = 350 + 100;
  *dt = c.cfl * std::fmin(std::fmin(c.dx, c.dy), c.dz) / maxwave;
  return PU_OK;
}

int pu_dycore_load_state(pu_dycore *h, const pu_state_view *coupler) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->load_state(coupler);
}

int pu_dycore_store_state(pu_dycore *h, pu_state_view *coupler) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->store_state(coupler);
}

int pu_dycore_advance(pu_dycore *h, double dt_dyn, int nsteps) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  if (!(dt_dyn > 0) || nsteps < 0) return fail(PU_ERR_INVALID, "dt must be positive and nsteps non-negative");
  PU_DEVICE_GUARD(h->device);
  return h->impl->advance(dt_dyn, nsteps);
}

int pu_dycore_time_step(pu_dycore *h, pu_state_view *coupler, double dt_phys, int *ncycles) {
  if (!h || !coupler) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  if (!(dt_phys > 0)) return fail(PU_ERR_INVALID, "dt_phys must be positive");
  PU_DEVICE_GUARD(h->device);
  double dt_dyn;
  pu_dycore_compute_time_step(h, &dt_dyn);
  const int n = (int)std::ceil(dt_phys / dt_dyn);
  dt_dyn = dt_phys / n;
  pu::NvtxRange range("pu_dycore_time_step");
  const int rc = h->impl->time_step(coupler, dt_dyn, n);
  if (ncycles) *ncycles = n;
  return rc;
}

int pu_dycore_get_conserved(pu_dycore *h, double *state, double *tracers, int mem) {
  if (!h || !state) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->get_conserved(state, tracers, mem);
}

int pu_dycore_set_conserved(pu_dycore *h, const double *state, const double *tracers, int mem) {
  if (!h || !state || !tracers) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->set_conserved(state, tracers, mem);
}

int pu_dycore_get_hydrostasis(pu_dycore *h, double *dc, double *tc, double *pc, double *de, double *te, double *pe) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  auto &I = *h->impl;
  const int nzh = I.nzh, ne = I.cfg.nz + 1;
  double *dst_c[3] = {dc, tc, pc}, *dst_e[3] = {de, te, pe};
  for (int q = 0; q < 3; q++) {
    if (dst_c[q] && cudaMemcpyAsync(dst_c[q], I.cells + q * nzh, nzh * sizeof(double), cudaMemcpyDeviceToHost, I.st))
      return fail(PU_ERR_CUDA, "copy of hydrostatic profiles failed");
    if (dst_e[q] && cudaMemcpyAsync(dst_e[q], I.edges + q * ne, ne * sizeof(double), cudaMemcpyDeviceToHost, I.st))
      return fail(PU_ERR_CUDA, "copy of hydrostatic profiles failed");
  }
  if (cudaStreamSynchronize(I.st) != cudaSuccess) return fail(PU_ERR_CUDA, "stream synchronize failed");
  return PU_OK;
}

int pu_dycore_set_hydrostasis(pu_dycore *h, const double *dens, const double *theta, const double *pressure) {
  if (!h || !dens || !theta || !pressure) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->set_hydrostasis(dens, theta, pressure);
}

int pu_dycore_diagnostics(pu_dycore *h, pu_diag *out) {
  if (!h || !out) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->diagnostics(out);
}

int pu_dycore_perturbations(pu_dycore *h, const pu_state_view *v, double *density_pert, double *theta_pert,
                            double *pressure_pert, int mem) {
  if (!h || !v || !density_pert || !theta_pert || !pressure_pert) return fail(PU_ERR_INVALID, "null argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->perturbations(v, density_pert, theta_pert, pressure_pert, mem);
}

int pu_dycore_synchronize(pu_dycore *h) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  PU_DEVICE_GUARD(h->device);
  return h->impl->check_err();
}

long long pu_dycore_kernel_launches(const pu_dycore *h) { return h ? h->impl->launches : 0; }

int pu_dycore_learned_harvest(pu_dycore *h, long long n, unsigned long long seed) {
  if (!h || n <= 0) return fail(PU_ERR_INVALID, "bad argument");
  if (!h->impl->inited) return fail(PU_ERR_STATE, "pu_dycore_init has not been called");
  PU_DEVICE_GUARD(h->device);
  return h->impl->ml_harvest(long(n), seed);
}

int pu_dycore_learned_train(pu_dycore *h, int steps, int batch, double lr, unsigned long long seed,
                            pu_learn_stats *out) {
  if (!h || steps < 0 || batch <= 0 || !(lr > 0)) return fail(PU_ERR_INVALID, "bad argument");
  PU_DEVICE_GUARD(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_train(steps, batch, lr, seed, out);
}

int pu_dycore_learned_get_weights(pu_dycore *h, float *theta) {
  if (!h || !theta) return fail(PU_ERR_INVALID, "null argument");
  PU_DEVICE_GUARD(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_get(theta);
}

int pu_dycore_learned_set_weights(pu_dycore *h, const float *theta) {
  if (!h || !theta) return fail(PU_ERR_INVALID, "null argument");
  PU_DEVICE_GUARD(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_set(theta);
}

int pu_dycore_learned_eval(pu_dycore *h, const float *x, long long n, float *wl, float *wr, int use_mma) {
  if (!h || !x || !wl || n <= 0) return fail(PU_ERR_INVALID, "bad argument");
  PU_DEVICE_GUARD(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_eval(x, long(n), wl, wr, use_mma);
}

int pu_dycore_learned_gradient(pu_dycore *h, const float *x, const float *t, long long n, float *grad,
                               double *loss) {
  if (!h || !x || !t || !grad || n <= 0 || n > (1 << 20)) return fail(PU_ERR_INVALID, "bad argument");
  PU_DEVICE_GUARD(h->device);
  int rc = h->impl->ml_alloc();
  if (rc) return rc;
  return h->impl->ml_gradient(x, t, long(n), grad, loss);
}

int pu_dycore_set_weno_mode(pu_dycore *h, int mode) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (mode != PU_WENO_PLAIN && mode != PU_WENO_LEARNED) return fail(PU_ERR_INVALID, "bad WENO mode");
  if (mode == PU_WENO_LEARNED) {
    if (h->impl->dc.on) return fail(PU_ERR_UNSUPPORTED, "learned weights do not run on decomposed tiles");
    if (h->impl->cfg.precision != PU_F32) return fail(PU_ERR_UNSUPPORTED, "learned weights run in the FP32 build only");
    if (!h->impl->cfg.weno_all)
      return fail(PU_ERR_UNSUPPORTED, "learned weights replace the limiter of weno_all; this dycore uses linear edges");
    if (!h->impl->ml_ready) return fail(PU_ERR_STATE, "learned weights are neither trained nor loaded");
  }
  h->impl->weno_mode = mode;
  return PU_OK;
}

int pu_dycore_learned_set_threshold(pu_dycore *h, double max_jump) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  if (!(max_jump >= 0)) return fail(PU_ERR_INVALID, "the jump threshold must be >= 0");
  h->impl->ml_jump = float(max_jump);
  return PU_OK;
}

int pu_dycore_learned_counts(pu_dycore *h, long long *learned, long long *fallback) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  PU_DEVICE_GUARD(h->device);
  unsigned long long c[2] = {0, 0};
  auto &I = *h->impl;
  if (I.ml_counts) {
    if (cudaMemcpyAsync(c, I.ml_counts, sizeof(c), cudaMemcpyDeviceToHost, I.st) != cudaSuccess ||
        cudaMemsetAsync(I.ml_counts, 0, sizeof(c), I.st) != cudaSuccess || cudaStreamSynchronize(I.st) != cudaSuccess)
      return fail(PU_ERR_CUDA, "reading the learned-path counters failed");
  }
  if (learned) *learned = (long long)c[0];
  if (fallback) *fallback = (long long)c[1];
  return PU_OK;
}

int pu_dycore_profile(pu_dycore *h, int enable) {
  if (!h) return fail(PU_ERR_INVALID, "null handle");
  PU_DEVICE_GUARD(h->device);
  if (cudaStreamSynchronize(h->impl->st) != cudaSuccess) return fail(PU_ERR_CUDA, "stream synchronize failed");
  h->impl->prof_reset();
  h->impl->profiling = enable != 0;
  return PU_OK;
}

int pu_dycore_profile_read(pu_dycore *h, pu_profile *out) {
  if (!h || !out) return fail(PU_ERR_INVALID, "null argument");
  PU_DEVICE_GUARD(h->device);
  return h->impl->prof_read(out);
}

int pu_decomp_process_grid(int nranks, long long nx_glob, long long ny_glob, int *nproc_x, int *nproc_y) {
  if (nranks < 1 || nx_glob < 1 || ny_glob < 1 || !nproc_x || !nproc_y) return fail(PU_ERR_INVALID, "bad argument");
  process_grid(nranks, nx_glob, ny_glob, *nproc_x, *nproc_y);
  return PU_OK;
}

int pu_decomp_tile(long long n_glob, int nproc, int p, long long *beg, long long *n) {
  if (n_glob < 1 || nproc < 1 || p < 0 || p >= nproc || !beg || !n) return fail(PU_ERR_INVALID, "bad argument");
  tile_range(n_glob, nproc, p, *beg, *n);
  return PU_OK;
}

int pu_decomp_neighbors(const pu_decomp *d, int nbr[4]) {
  if (!d || !nbr || d->nproc_x < 1 || d->nproc_y < 1) return fail(PU_ERR_INVALID, "bad argument");
  neighbors(*d, nbr);
  return PU_OK;
}

int pu_nccl_get_unique_id(unsigned char *id) {
  if (!id) return fail(PU_ERR_INVALID, "null argument");
  auto &api = pu::nccl();
  if (!api.ok) return fail(PU_ERR_UNSUPPORTED, api.error);
  ncclUniqueId u;
  const ncclResult_t r = api.GetUniqueId(&u);
  if (r != ncclSuccess) return fail(PU_ERR_CUDA, std::string("ncclGetUniqueId: ") + api.GetErrorString(r));
  static_assert(sizeof(u.internal) == PU_NCCL_ID_BYTES, "NCCL unique id size");
  std::memcpy(id, u.internal, PU_NCCL_ID_BYTES);
  return PU_OK;
}

int pu_dycore_set_decomposition(pu_dycore *h, const pu_decomp *d, const unsigned char *nccl_id) {
  if (!h || !d) return fail(PU_ERR_INVALID, "null argument");
  auto &I = *h->impl;
  if (I.inited) return fail(PU_ERR_STATE, "pu_dycore_set_decomposition comes before pu_dycore_init");
  if (I.dc.on) return fail(PU_ERR_STATE, "the handle is already decomposed");
  if (I.weno_mode == PU_WENO_LEARNED) return fail(PU_ERR_UNSUPPORTED, "learned weights do not run on decomposed tiles");
  int rc = check_decomp(d, I.cfg);
  if (rc) return rc;
  PU_DEVICE_GUARD(h->device);
  rc = set_decomposition(I, *d, nccl_id);
  if (rc) I.dec_release();
  return rc;
}

int pu_dycore_set_decomposition_host(pu_dycore *h, const pu_decomp *d, const pu_host_transport *t) {
  if (!h || !d || !t) return fail(PU_ERR_INVALID, "null argument");
  if (!t->exchange || !t->allreduce_sum_f64 || !t->allgather)
    return fail(PU_ERR_INVALID, "the host transport needs exchange, allreduce_sum_f64 and allgather");
  auto &I = *h->impl;
  if (I.inited) return fail(PU_ERR_STATE, "pu_dycore_set_decomposition_host comes before pu_dycore_init");
  if (I.dc.on) return fail(PU_ERR_STATE, "the handle is already decomposed");
  if (I.weno_mode == PU_WENO_LEARNED) return fail(PU_ERR_UNSUPPORTED, "learned weights do not run on decomposed tiles");
  int rc = check_decomp(d, I.cfg);
  if (rc) return rc;
  PU_DEVICE_GUARD(h->device);
  rc = set_decomposition(I, *d, nullptr);
  if (!rc) {
    // Every rank checks the whole table of tiles before any halo moves.
    const TileInfo mine{d->px, d->py, I.cfg.nx, I.cfg.ny, I.cfg.nz, I.S, I.cfg.precision};
    std::vector<TileInfo> all(I.dc.nranks);
    const int q = t->allgather(t->user, &mine, all.data(), sizeof(TileInfo));
    std::string why;
    if (q != 0) rc = fail(PU_ERR_TRANSPORT, "host transport: allgather returned " + std::to_string(q));
    else if (!tiles_fit(*d, all, why)) rc = fail(PU_ERR_INVALID, why);
  }
  if (rc) {
    I.dec_release();
    I.dc.on = false;
    return rc;
  }
  I.dc.host = true;
  I.dc.ht = *t;
  return PU_OK;
}

int pu_dycore_group_init(pu_dycore *const *hs, int n, const pu_state_view *views, const double *const *props,
                         const double *const *projs, int mem) {
  std::vector<pu::ImplBase *> t;
  int rc = group_tiles(hs, n, t, false);
  if (rc) return rc;
  if (!views) return fail(PU_ERR_INVALID, "null views");
  PU_DEVICE_GUARD(hs[0]->device);
  for (int i = 0; i < n; i++) {
    rc = hs[i]->impl->dinit_begin(&views[i], props ? props[i] : nullptr, projs ? projs[i] : nullptr, mem);
    if (rc) return rc;
  }
  // Profile sums over the tiles in rank order, with compensation.
  const int nz = t[0]->cfg.nz;
  std::vector<double> part(size_t(3) * nz), sum(size_t(3) * nz, 0.0), comp(size_t(3) * nz, 0.0);
  for (pu::ImplBase *a : t) {
    if (cudaMemcpyAsync(part.data(), a->sums, part.size() * sizeof(double), cudaMemcpyDeviceToHost, a->st) !=
            cudaSuccess ||
        cudaStreamSynchronize(a->st) != cudaSuccess)
      return fail(PU_ERR_CUDA, "profile sums copy failed");
    for (size_t q = 0; q < part.size(); q++) {
      const double x = part[q], tq = sum[q] + x;
      comp[q] += std::fabs(sum[q]) >= std::fabs(x) ? (sum[q] - tq) + x : (x - tq) + sum[q];
      sum[q] = tq;
    }
  }
  for (size_t q = 0; q < sum.size(); q++) sum[q] += comp[q];
  for (pu::ImplBase *a : t)
    if ((rc = a->dinit_hydro(sum.data()))) return rc;
  if ((rc = local_exchange(t, 1, true, false))) return rc;
  for (pu::ImplBase *a : t)
    if ((rc = a->dinit_mid())) return rc;
  if (!t[0]->sim2d() && (rc = local_exchange(t, 2, false, true))) return rc;
  for (int i = 0; i < n; i++)
    if ((rc = hs[i]->impl->dinit_end(&views[i]))) return rc;
  return PU_OK;
}

int pu_dycore_group_advance(pu_dycore *const *hs, int n, double dt, int nsteps) {
  std::vector<pu::ImplBase *> t;
  int rc = group_tiles(hs, n, t, true);
  if (rc) return rc;
  if (!(dt > 0)) return fail(PU_ERR_INVALID, "dt must be positive");
  if (nsteps <= 0) return PU_OK;
  PU_DEVICE_GUARD(hs[0]->device);
  for (pu::ImplBase *a : t)
    if ((rc = a->dec_enforce())) return rc;
  for (int s = 0; s < nsteps; s++)
    for (int sg = 0; sg < 3; sg++) {
      for (pu::ImplBase *a : t)
        if ((rc = a->dec_pack(sg))) return rc;
      if ((rc = local_exchange(t, 0, true, !t[0]->sim2d()))) return rc;
      for (pu::ImplBase *a : t)
        if ((rc = a->dec_compute(sg, dt, s == nsteps - 1))) return rc;
    }
  return PU_OK;
}

int pu_dycore_group_time_step(pu_dycore *const *hs, int n, pu_state_view *views, double dt_phys, int *ncycles) {
  std::vector<pu::ImplBase *> t;
  int rc = group_tiles(hs, n, t, true);
  if (rc) return rc;
  if (!views) return fail(PU_ERR_INVALID, "null views");
  if (!(dt_phys > 0)) return fail(PU_ERR_INVALID, "dt_phys must be positive");
  PU_DEVICE_GUARD(hs[0]->device);
  double dt_dyn;
  pu_dycore_compute_time_step(hs[0], &dt_dyn);
  const int nc = (int)std::ceil(dt_phys / dt_dyn);
  dt_dyn = dt_phys / nc;
  for (int i = 0; i < n; i++)
    if ((rc = hs[i]->impl->load_state(&views[i]))) return rc;
  if ((rc = pu_dycore_group_advance(hs, n, dt_dyn, nc))) return rc;
  for (int i = 0; i < n; i++)
    if ((rc = hs[i]->impl->store_state(&views[i]))) return rc;
  if (ncycles) *ncycles = nc;
  return PU_OK;
}

int pu_weno9_edges_f32(const float *stencils, const unsigned char *flags, long long n, int variant, float *qL,
                       float *qR, int mem) {
  if (!stencils || !qL || !qR || n < 0 || variant < 0 || variant > 4) return fail(PU_ERR_INVALID, "bad argument");
  if (n == 0) return PU_OK;
  const bool dev = pu::resolve_mem(mem, stencils) == PU_MEM_DEVICE;
  float *ds = const_cast<float *>(stencils), *dl = qL, *dr = qR;
  unsigned char *df = const_cast<unsigned char *>(flags);
  if (!dev) {
    if (cudaMalloc(&ds, size_t(n) * 9 * sizeof(float)) != cudaSuccess) return fail(PU_ERR_NOMEM, "cudaMalloc");
    cudaMalloc(&dl, size_t(n) * sizeof(float));
    cudaMalloc(&dr, size_t(n) * sizeof(float));
    if (flags) cudaMalloc(&df, size_t(n));
    cudaMemcpy(ds, stencils, size_t(n) * 9 * sizeof(float), cudaMemcpyHostToDevice);
    if (flags) cudaMemcpy(df, flags, size_t(n), cudaMemcpyHostToDevice);
  }
  const long long threads = variant == 0 ? n : (n + 1) / 2;
  const unsigned blocks = unsigned((threads + 255) / 256);
  int *derr = nullptr;
  if (variant == 0) k_weno9_eval<0><<<blocks, 256>>>(ds, df, n, dl, dr);
  else if (variant == 1) k_weno9_eval<1><<<blocks, 256>>>(ds, df, n, dl, dr);
  else if (variant == 4) k_weno9_eval<4><<<blocks, 256>>>(ds, df, n, dl, dr);
  else {
    if (cudaMalloc(&derr, sizeof(int)) == cudaSuccess) {
      cudaMemset(derr, 0, sizeof(int));
      const long long nb = (n + 127) / 128;
      if (variant == 2) {
        k_weno9_tc<<<unsigned(nb < 148 * 8 ? nb : 148 * 8), 128>>>(ds, df, n, dl, dr, derr);
      } else {
        const long long nb2 = (n + 255) / 256;
        k_weno9_tc_ts<<<unsigned(nb2 < 148 * 4 ? nb2 : 148 * 4), 256>>>(ds, df, n, dl, dr, derr);
      }
    }
  }
  cudaError_t e = cudaGetLastError();
  if (e == cudaSuccess) e = cudaDeviceSynchronize();
  int herr = 0;
  if (derr) {
    cudaMemcpy(&herr, derr, sizeof(int), cudaMemcpyDeviceToHost);
    cudaFree(derr);
  }
  if (!dev) {
    if (e == cudaSuccess) {
      cudaMemcpy(qL, dl, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost);
      cudaMemcpy(qR, dr, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost);
    }
    cudaFree(ds);
    cudaFree(dl);
    cudaFree(dr);
    if (df) cudaFree(df);
  }
  if (e != cudaSuccess) return fail(PU_ERR_CUDA, cudaGetErrorString(e));
  if (herr) return fail(PU_ERR_CUDA, "tensor-core limiter: an MMA did not complete in time");
  return PU_OK;
}

int pu_learned_normalize_f32(const float *stencils, long long n, float *x, float *jump) {
  if (!stencils || !x || !jump || n < 0) return fail(PU_ERR_INVALID, "bad argument");
  if (n == 0) return PU_OK;
  float *ds = nullptr, *dx = nullptr, *dj = nullptr;
  if (cudaMalloc(&ds, size_t(n) * 9 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&dx, size_t(n) * 9 * sizeof(float)) != cudaSuccess ||
      cudaMalloc(&dj, size_t(n) * sizeof(float)) != cudaSuccess) {
    cudaFree(ds);
    cudaFree(dx);
    return fail(PU_ERR_NOMEM, "cudaMalloc");
  }
  cudaError_t e = cudaMemcpy(ds, stencils, size_t(n) * 9 * sizeof(float), cudaMemcpyHostToDevice);
  if (e == cudaSuccess) {
    k_normalize9_eval<<<unsigned((n + 255) / 256), 256>>>(ds, n, dx, dj);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaMemcpy(x, dx, size_t(n) * 9 * sizeof(float), cudaMemcpyDeviceToHost);
  if (e == cudaSuccess) e = cudaMemcpy(jump, dj, size_t(n) * sizeof(float), cudaMemcpyDeviceToHost);
  cudaFree(ds);
  cudaFree(dx);
  cudaFree(dj);
  if (e != cudaSuccess) return fail(PU_ERR_CUDA, cudaGetErrorString(e));
  return PU_OK;
}

int pu_check_bounded_wait(int limit_us, int *completed, double *ms, long long *cycles) {
  if (limit_us < 0 || limit_us > 1000000 || !completed) return fail(PU_ERR_INVALID, "bad argument");
  const unsigned long long limit_ns = limit_us ? 1000ull * limit_us : pu::tma::WAIT_LIMIT_NS;
  long long *d = nullptr, h[2] = {0, 0};
  if (cudaMalloc(&d, sizeof(h)) != cudaSuccess) return fail(PU_ERR_NOMEM, "cudaMalloc");
  cudaEvent_t e0 = nullptr, e1 = nullptr;
  cudaError_t e = cudaEventCreate(&e0);
  if (e == cudaSuccess) e = cudaEventCreate(&e1);
  if (e == cudaSuccess) e = cudaEventRecord(e0);
  if (e == cudaSuccess) {
    k_wait_check<<<1, 128>>>(limit_ns, d);
    e = cudaGetLastError();
  }
  if (e == cudaSuccess) e = cudaEventRecord(e1);
  if (e == cudaSuccess) e = cudaMemcpy(h, d, sizeof(h), cudaMemcpyDeviceToHost);
  float t = 0.f;
  if (e == cudaSuccess) e = cudaEventElapsedTime(&t, e0, e1);
  if (e0) cudaEventDestroy(e0);
  if (e1) cudaEventDestroy(e1);
  cudaFree(d);
  if (e != cudaSuccess) return fail(PU_ERR_CUDA, cudaGetErrorString(e));
  *completed = int(h[0]);
  if (ms) *ms = t;
  if (cycles) *cycles = h[1];
  return PU_OK;
}

}  // extern "C"
