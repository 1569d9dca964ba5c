// noalloc.cu — a forward entry point that allocates no device memory.
//
// Who needs it: callers that must not call cudaMalloc while they run — a host that has handed
// all device memory to its own pool or arena and forbids allocations outside it, a real-time or
// embedded pipeline that pre-allocates everything at start-up so no call can stall or fail on an
// allocation, or code running where allocation is not permitted.  For them this entry computes the
// same noiseless, spike-free forward as `mrsim_build_coil_kspaces` (the existing kernels, launched
// unchanged) but keeps every piece of intermediate device memory in file-scope `static __device__`
// arrays: the y-stage output that the x-stage reads (the scratch), the static-phase plane, and
// the staged geometry tables, line table, unit descriptor and tile lists.  The caller passes
// device pointers for the inputs and the output.
//
// Costs and rules:
//  - every GPU that loads the library holds these arrays (about 7.8 MiB) until the process exits;
//  - the sizes are capped (see the limits below); larger slices are rejected with an error;
//  - the first call on a device resolves the arrays' device addresses with cudaGetSymbolAddress
//    (with that device current) and caches them with the identity of the device's current CUDA
//    context; a later call in another context (after cudaDeviceReset, say) resolves them again;
//  - every call checks that its data pointers are device (or managed) memory of the current
//    device, so a host pointer passed by mistake is an error, not a device fault;
//  - each call waits for its stream before it returns (the host tables it stages must outlive
//    their copies);
//  - every call shares the arrays, which keep the last call's contents: calls that overlap on
//    the GPU (two streams, or two host threads) race on them and must be serialised by the caller.
#include <cuda.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <mutex>
#include <vector>

#include "driver.h"
#include "host_tables.h"
#include "mrsim_internal.h"

namespace mrsim {
namespace {

// limits of the static arrays
constexpr size_t kNaScratch = size_t(1) << 19;  // float2: ncoils * acquired lines * snx
constexpr size_t kNaPlane = size_t(1) << 18;    // float: snx * sny
constexpr size_t kNaTw = size_t(1) << 18;       // float2: 4 * snx * nx
constexpr size_t kNaAxis = size_t(1) << 15;     // float: ncoils * snx, ncoils * sny
constexpr size_t kNaLines = 1024;
constexpr size_t kNaTiles = 8192;
constexpr size_t kNaXTiles = 2048;

static __device__ __align__(256) float2 na_scratch[kNaScratch];
static __device__ __align__(256) float na_phase[kNaPlane];
static __device__ __align__(256) float2 na_tw[kNaTw];
static __device__ __align__(256) float na_ex[kNaAxis];
static __device__ __align__(256) float na_ey[kNaAxis];
static __device__ __align__(256) LineRec na_lines[kNaLines];
static __device__ __align__(256) UnitDesc na_unit[1];
static __device__ __align__(256) StaticDesc na_static[1];
static __device__ __align__(256) int4 na_ytiles[kNaTiles];
static __device__ __align__(256) XTile na_xtiles[kNaXTiles];

struct NaAddrs {
  float2* scratch = nullptr;
  float* phase = nullptr;
  float2* tw = nullptr;
  float* ex = nullptr;
  float* ey = nullptr;
  LineRec* lines = nullptr;
  UnitDesc* unit = nullptr;
  StaticDesc* statics = nullptr;
  int4* ytiles = nullptr;
  XTile* xtiles = nullptr;
  unsigned long long ctx_id = 0;
  bool ready = false;
};

constexpr int kMaxDevices = 64;
NaAddrs g_addrs[kMaxDevices];
std::mutex g_addr_mu;

// The identity of the calling thread's current CUDA context (0 when it cannot be told): the
// driver's cuCtxGetCurrent / cuCtxGetId, reached through the runtime's entry-point query so that
// the library needs no link against the driver library.
unsigned long long current_context_id() {
  using GetCurrent = CUresult (*)(CUcontext*);
  using GetId = CUresult (*)(CUcontext, unsigned long long*);
  static GetCurrent get_current = nullptr;
  static GetId get_id = nullptr;
  static std::once_flag once;
  std::call_once(once, [] {
    void* f = nullptr;
    cudaDriverEntryPointQueryResult q;
    if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_current = (GetCurrent)f;
    f = nullptr;
    if (cudaGetDriverEntryPoint("cuCtxGetId", &f, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      get_id = (GetId)f;
  });
  if (!get_current || !get_id) return 0;
  CUcontext c = nullptr;
  unsigned long long id = 0;
  if (get_current(&c) != CUDA_SUCCESS || !c || get_id(c, &id) != CUDA_SUCCESS) return 0;
  return id;
}

// Set-up, once per device (and again if the device's context changed), with that device
// current: the arrays' device addresses.
const NaAddrs& addresses(int device) {
  std::lock_guard<std::mutex> lk(g_addr_mu);
  NaAddrs& a = g_addrs[device];
  const unsigned long long id = current_context_id();
  if (!a.ready || a.ctx_id != id) {
    a.ready = false;
    void* p = nullptr;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_scratch));
    a.scratch = (float2*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_phase));
    a.phase = (float*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_tw));
    a.tw = (float2*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_ex));
    a.ex = (float*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_ey));
    a.ey = (float*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_lines));
    a.lines = (LineRec*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_unit));
    a.unit = (UnitDesc*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_static));
    a.statics = (StaticDesc*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_ytiles));
    a.ytiles = (int4*)p;
    MRSIM_CUDA(cudaGetSymbolAddress(&p, na_xtiles));
    a.xtiles = (XTile*)p;
    a.ctx_id = id;
    a.ready = true;
  }
  return a;
}

// A data pointer the kernels will read or write must be device (or managed) memory that the
// current device can reach; cudaPointerGetAttributes allocates nothing.
void need_device_pointer(const void* p, const char* what, int device) {
  if (!p) fail(std::string("mrsim_build_coil_kspaces_noalloc: ") + what + " is NULL");
  cudaPointerAttributes at;
  std::memset(&at, 0, sizeof at);
  cudaError_t e = cudaPointerGetAttributes(&at, p);
  if (e != cudaSuccess) {
    (void)cudaGetLastError();  // clear the (non-sticky) error the query left behind
    fail(std::string("mrsim_build_coil_kspaces_noalloc: ") + what + " is not a device pointer");
  }
  const bool ok = (at.type == cudaMemoryTypeDevice && at.device == device) || at.type == cudaMemoryTypeManaged;
  if (!ok)
    fail(std::string("mrsim_build_coil_kspaces_noalloc: ") + what +
         " must be device memory of the current device (host memory was passed)");
}

void too_big(const char* what, size_t need, size_t cap) {
  fail(std::string("mrsim_build_coil_kspaces_noalloc: ") + what + " needs " + std::to_string(need) +
       " elements, above the static limit of " + std::to_string(cap));
}

}  // namespace

void build_coil_kspaces_noalloc(const mrsim_slice_input& inp, const mrsim_acquisition& acq, float2* out,
                                cudaStream_t st) {
  const int snx = (int)inp.sim[0], sny = (int)inp.sim[1], nx = (int)inp.acq_matrix[0], ny = (int)inp.acq_matrix[1];
  if (snx <= 0 || sny <= 0 || nx <= 0 || ny <= 0) fail("empty simulation grid or acquired matrix");
  if (!(snx % nx == 0 && sny % ny == 0)) fail("sim grid must be an integer multiple of the acquired matrix");
  const int ncomp = (int)inp.ncomp;
  if (ncomp > kMaxComp) fail("more than 8 compartments");
  const int ncoils = (int)std::max<int64_t>(acq.n_coils, 1);
  if (ncoils > kMaxCoils) fail("more than 64 coils");
  bool uniform = true;
  for (int c = 0; c < ncomp; ++c) uniform = uniform && !inp.t2[c].is_map;
  if (inp.t_inhom)
    for (int c = 0; c < ncomp; ++c) uniform = uniform && !inp.t_inhom[c].is_map;
  if (!uniform) fail("mrsim_build_coil_kspaces_noalloc: T2/T2' maps are not supported (uniform values only)");
  int dev = 0;
  MRSIM_CUDA(cudaGetDevice(&dev));
  if (dev < 0 || dev >= kMaxDevices) fail("device ordinal out of range");
  // every pointer a kernel dereferences: device memory of this device, checked before any copy
  for (int c = 0; c < ncomp; ++c) need_device_pointer(inp.compartments[c], "a compartment plane", dev);
  need_device_pointer(inp.fmap, "fmap", dev);
  if (inp.phase0) need_device_pointer(inp.phase0, "phase0", dev);
  need_device_pointer(out, "kspace", dev);
  if (ncomp > 1)
    for (int c = 1; c < ncomp; ++c)
      if (inp.compartments[c] != inp.compartments[0] + (size_t)c * snx * sny)
        fail("mrsim_build_coil_kspaces_noalloc: compartment planes must be contiguous on the device");
  const NaAddrs& A = addresses(dev);

  const bool eddy = acq.eddy_strength != 0.0 && inp.has_eddy_drive;
  const bool eddy_phase = acq.eddy_phase != 0.0 && inp.has_eddy_drive;
  float t2u[kMaxComp], tiu[kMaxComp];
  for (int c = 0; c < kMaxComp; ++c) {
    t2u[c] = c < ncomp ? inp.t2[c].value : 1.f;
    tiu[c] = c < ncomp ? (inp.t_inhom ? inp.t_inhom[c].value : (float)acq.t_inhom) : 1.f;
  }
  LineTimingTab lt = line_timing(acq, nx, ny);
  std::vector<LineRec> lines;
  // the per-line factors of `build_coil_kspace_timed` (kspace.rs:843-903)
  {
    auto mask = sampling_mask(nx, ny, acq);
    for (int ky = 0; ky < ny; ++ky) {
      if (!mask[(size_t)nx * ky]) continue;
      LineRec L;
      std::memset(&L, 0, sizeof L);
      L.ky = ky;
      L.row = ky;
      L.pol = lt.polarity[ky] < 0 ? -1 : 1;
      const double t = lt.t_ms[ky] / 1000.0, trf = lt.trf_ms[ky];
      const bool spin = acq.echo == MRSIM_ECHO_SPIN;
      const double tb0 = spin ? t : t + acq.t_echo / 1000.0;
      L.t_hi = (float)tb0;
      L.t_lo = (float)(tb0 - (double)L.t_hi);
      L.t_s = (float)tb0;
      const double inh = spin ? std::fabs(t) * 1000.0 : trf;
      L.inhom_ms = (float)inh;
      L.trf_ms = (float)trf;
      L.decay = eddy ? (float)(std::exp(-lt.tread_ms[ky] / acq.eddy_tau) * t) : 0.f;
      for (int c = 0; c < kMaxComp; ++c) {
        double rel = 1.0;
        if (c < ncomp && acq.do_relaxation)
          rel = std::exp(-trf / (double)t2u[c] - inh / (inp.t_inhom ? (double)tiu[c] : acq.t_inhom));
        L.rel[c] = (float)rel;
      }
      lines.push_back(L);
    }
  }
  const size_t nl = lines.size();
  if (nl > kNaLines) too_big("the line table", nl, kNaLines);
  if ((size_t)ncoils * nl * snx > kNaScratch) too_big("the y-stage scratch", (size_t)ncoils * nl * snx, kNaScratch);
  if ((size_t)snx * sny > kNaPlane) too_big("the static-phase plane", (size_t)snx * sny, kNaPlane);
  if ((size_t)4 * snx * nx > kNaTw) too_big("the x-stage twiddles", (size_t)4 * snx * nx, kNaTw);
  if ((size_t)ncoils * std::max(snx, sny) > kNaAxis)
    too_big("the coil tables", (size_t)ncoils * std::max(snx, sny), kNaAxis);

  // geometry tables, as `build_geo` computes them, staged into the static arrays
  const int ox = snx / nx, oy = sny / ny;
  const double xoff = (ox - 1.0) / 2.0, yoff = (oy - 1.0) / 2.0;
  const int xs = nx / 2, sxs = ox * xs;
  std::vector<float> ex((size_t)ncoils * snx, 1.f), ey((size_t)ncoils * sny, 1.f);
  if (ncoils > 1) {
    const double sigma = 0.9 * (double)std::max(nx, ny), r = 0.6 * (double)std::max(nx, ny);
    for (int q = 0; q < ncoils; ++q) {
      const double ang = kTau * (double)q / (double)ncoils;
      const double px = nx / 2.0 + r * std::cos(ang), py = ny / 2.0 + r * std::sin(ang);
      for (int x = 0; x < snx; ++x) {
        double d = ((double)x - xoff) / ox - px;
        ex[(size_t)q * snx + x] = (float)std::exp(-(d * d) / (2.0 * sigma * sigma));
      }
      for (int y = 0; y < sny; ++y) {
        double d = ((double)y - yoff) / oy - py;
        ey[(size_t)q * sny + y] = (float)std::exp(-(d * d) / (2.0 * sigma * sigma));
      }
    }
  }
  std::vector<float2> tw((size_t)4 * snx * nx);
  const double c0 = (double)sxs + xoff;
  const long long m2 = 2LL * snx;
  for (int pol = 0; pol < 2; ++pol) {
    const double gh = pol == 0 ? acq.ghost_offset : -acq.ghost_offset;
    for (int x = 0; x < snx; ++x) {
      const long long X = 2LL * (x - sxs) - (ox - 1);
      const double gramp = gh * ((double)x - c0) / (double)snx;
      for (int kx = 0; kx < nx; ++kx) {
        double turns = (double)(((long long)(kx - xs) * X) % m2) / (double)m2 + gramp;
        turns -= std::rint(turns);
        float2 v = make_float2((float)std::cos(kTau * turns), (float)std::sin(kTau * turns));
        tw[(size_t)pol * snx * nx + (size_t)x * nx + kx] = v;
        tw[(size_t)(2 + pol) * snx * nx + (size_t)kx * snx + x] = v;
      }
    }
  }
  MRSIM_CUDA(cudaMemcpyAsync(A.ex, ex.data(), ex.size() * 4, cudaMemcpyHostToDevice, st));
  MRSIM_CUDA(cudaMemcpyAsync(A.ey, ey.data(), ey.size() * 4, cudaMemcpyHostToDevice, st));
  MRSIM_CUDA(cudaMemcpyAsync(A.tw, tw.data(), tw.size() * sizeof(float2), cudaMemcpyHostToDevice, st));
  if (nl) MRSIM_CUDA(cudaMemcpyAsync(A.lines, lines.data(), nl * sizeof(LineRec), cudaMemcpyHostToDevice, st));

  StaticDesc sd;
  std::memset(&sd, 0, sizeof sd);
  sd.snx = snx;
  sd.sny = sny;
  sd.nx = nx;
  sd.ny = ny;
  sd.o = ox;
  sd.z = (int)inp.z;
  sd.nz_full = (int)inp.nz;
  sd.flags = (inp.phase0 ? 1 : 0) | (eddy_phase ? 2 : 0);
  sd.phase0 = inp.phase0;
  double grad[3] = {0, 0, 0};
  if (inp.has_eddy_drive)
    for (int i = 0; i < 3; ++i) grad[i] = inp.eddy_drive[i];
  for (int i = 0; i < 3; ++i) sd.eddy_phase_coef[i] = acq.eddy_phase * grad[i];
  sd.zc_c = (double)inp.z - ((double)inp.nz - 1.0) / 2.0;
  sd.out = A.phase;

  UnitDesc u;
  std::memset(&u, 0, sizeof u);
  u.snx = snx;
  u.sny = sny;
  u.nx = nx;
  u.ny = ny;
  u.ncomp = ncomp;
  u.ncoils = ncoils;
  u.n_lines = (int)nl;
  u.n_rows = ny;
  u.flags = (acq.do_relaxation ? UF_RELAX : 0) | (eddy ? UF_EDDY : 0) | (acq.do_distortions ? UF_DISTORT : 0) |
            (acq.echo == MRSIM_ECHO_GRADIENT ? UF_GRADIENT : 0);
  u.z = (int)inp.z;
  u.nz = (int)inp.nz;
  u.comp_stride = (long long)snx * sny;
  u.map_stride = (long long)snx * sny;
  u.comp = ncomp > 0 ? inp.compartments[0] : nullptr;
  u.fmap = inp.fmap;
  u.phase = A.phase;
  u.lines = A.lines;
  u.geo.ex = A.ex;
  u.geo.ey = A.ey;
  u.geo.tw = A.tw;
  u.geo.coil_off = ncoils <= 1 ? 0.f : 0.15f;
  u.signal_scale = (float)acq.signal_scale;
  for (int c = 0; c < kMaxComp; ++c) {
    u.t2u[c] = t2u[c];
    u.tiu[c] = tiu[c];
  }
  if (eddy) {
    const double zc = (double)inp.z - (double)(inp.nz / 2);
    u.eddy_cx = (float)(acq.eddy_strength * grad[0]);
    u.eddy_qx = (float)(acq.eddy_quad * grad[0]);
    u.eddy_cy = (float)(acq.eddy_strength * grad[1]);
    u.eddy_qy = (float)(acq.eddy_quad * grad[1]);
    u.eddy_z = (float)(acq.eddy_strength * grad[2] * zc + acq.eddy_quad * grad[2] * zc * zc);
  }
  u.kspace = out;
  u.g = A.scratch;
  MRSIM_CUDA(cudaMemcpyAsync(A.unit, &u, sizeof u, cudaMemcpyHostToDevice, st));
  MRSIM_CUDA(cudaMemcpyAsync(A.statics, &sd, sizeof sd, cudaMemcpyHostToDevice, st));

  // the tile lists of `epi_plan_create`, staged into the static arrays
  EpiPlan plan;  // a view over the static arrays: its `allocs` list stays empty, it frees nothing
  plan.n_units = 1;
  plan.d_units = A.unit;
  plan.n_statics = 1;
  plan.d_statics = A.statics;
  plan.max_static_n = snx * sny;
  plan.max_sny = sny;
  plan.max_snx = snx;
  plan.max_nx = nx;
  plan.max_lines = (int)nl;
  plan.max_coils = ncoils;
  plan.nc = ncomp <= 1 ? 1 : ncomp <= 2 ? 2 : ncomp <= 3 ? 3 : ncomp <= 4 ? 4 : 8;
  plan.qg = ncoils <= 1 ? 1 : ncoils <= 2 ? 2 : ncoils <= 4 ? 4 : 8;
  std::vector<int4> yt;
  std::vector<XTile> xt;
  for (int l = 0; l < (int)nl; l += 4)  // the y-stage covers 4 lines per CTA
    for (int x0 = 0; x0 < snx; x0 += 128)
      for (int q0 = 0; q0 < ncoils; q0 += plan.qg) yt.push_back(make_int4(0, l, x0, q0));
  append_xtiles(xt, u, 0, lines.data(), 0);
  if (yt.size() > kNaTiles) too_big("the y-stage tile list", yt.size(), kNaTiles);
  if (xt.size() > kNaXTiles) too_big("the x-stage tile list", xt.size(), kNaXTiles);
  if (!yt.empty()) MRSIM_CUDA(cudaMemcpyAsync(A.ytiles, yt.data(), yt.size() * sizeof(int4), cudaMemcpyHostToDevice, st));
  if (!xt.empty()) MRSIM_CUDA(cudaMemcpyAsync(A.xtiles, xt.data(), xt.size() * sizeof(XTile), cudaMemcpyHostToDevice, st));
  plan.d_ytiles[0] = A.ytiles;
  plan.n_ytiles[0] = (int)yt.size();
  plan.d_gtiles[0] = A.xtiles;
  plan.n_gtiles[0] = (int)xt.size();

  MRSIM_CUDA(cudaMemsetAsync(out, 0, sizeof(float2) * (size_t)ncoils * nx * ny, st));
  epi_plan_statics(&plan, st);
  if (nl) epi_plan_forward(&plan, st);
  // synchronous: the output is complete, and the staged host tables are no longer read, on return
  MRSIM_CUDA(cudaStreamSynchronize(st));
}

}  // namespace mrsim
