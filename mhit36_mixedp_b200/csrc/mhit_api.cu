// C ABI of libmhit_b200.so: context management, the per-step launch sequence, CUDA-graph
// replay, field/particle transfer, field files and the input.inp parser.
//
// One step (multi/main.f90:456-1007) is this launch sequence on the context stream:
//   [tracers] k_tracer                       :477-508
//   [phase]   k_phase                        :522-636
//             k_mom                          :658-816
//             k_div_fftx, k_fft_cols(y fwd),
//             k_fft_cols(z fwd+solve+inv),
//             k_fft_cols(y inv), k_fftx_inv  :833-923
//             k_correct, k_finalize          :942-1007
// Steps after the first are replayed from two captured CUDA graphs (one per parity of the
// velocity ping-pong buffers), so a step costs one graph launch on the host.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <algorithm>
#include <cstring>
#include <functional>
#include <string>
#include <vector>

#include "../../include/mhit_b200.h"
#include "common.cuh"
#include "kernels.h"

namespace mhit {

static thread_local std::string g_err;

int set_error(int code, const std::string& msg) {
  g_err = msg;
  return code;
}

int set_cuda_error(cudaError_t e, const char* expr, const char* file, int line) {
  char buf[512];
  snprintf(buf, sizeof(buf), "CUDA error %d (%s) in %s at %s:%d", (int)e, cudaGetErrorString(e), expr, file, line);
  g_err = buf;
  return MHIT_ERR_CUDA;
}

}  // namespace mhit

using namespace mhit;

enum {
  ST_TRACER = 0, ST_PHASE, ST_MOM, ST_XFWD, ST_YFWD, ST_ZSOLVE, ST_YINV, ST_XINV, ST_REFINE, ST_CORRECT, ST_COUNT
};
static const char* kStageNames[ST_COUNT] = {"k_tracer", "k_phase", "k_mom", "k_div_fftx", "k_fft_cols_yfwd",
                                            "k_fft_cols_zsolve", "k_fft_cols_yinv", "k_fftx_inv",
                                            "refine(5 passes)", "k_correct+k_finalize"};
static const char* kFusedCorrectName = "k_xinv_correct+k_finalize";

struct mhit_ctx {
  mhit_params prm;
  Geo g;
  int dev = 0;
  cudaStream_t st = nullptr;
  size_t n = 0;
  double *U[2] = {}, *V[2] = {}, *W[2] = {};
  double *RU = nullptr, *RV = nullptr, *RW = nullptr;
  double *PHI[2] = {}, *RPHI = nullptr;
  void* P = nullptr;
  float* Q[2] = {};       // incremental: the FP32 predictor, ping-pong (the step reading set k reads Q[k])
  float* P2 = nullptr;    // refinement: the pressure correction (FP32)
  double* P64 = nullptr;  // refinement: corrected pressure for a download; incremental: the pressure (FP64)
  double* Pw = nullptr;   // FP32 modes: the pressure widened to FP64 for a download (lazy)
  void* lab_small = nullptr;  // droplet labelling scratch (trig tables, chunk counts), grown lazily
  size_t lab_small_bytes = 0;
  void* lab_acc = nullptr;    // droplet labelling per-drop sums, grown lazily
  size_t lab_acc_bytes = 0;
  void* spec = nullptr;
  void *twx = nullptr, *twy = nullptr, *twz = nullptr;
  void* spec64 = nullptr;  // energy spectrum in the FP32 modes: an FP64 half spectrum, grown lazily
  size_t spec64_bytes = 0;
  void* tw64[3] = {};      // ... and FP64 twiddles
  double *k2x = nullptr, *k2y = nullptr, *k2z = nullptr;
  double* tabs = nullptr;
  double* partials = nullptr;
  int nblk = 0;
  DevScalars* sc = nullptr;
  DevScalars* sc_host = nullptr;
  double* part = nullptr;
  int np = 0;
  int cur = 0;
  long long nstep = 0;
  bool graph_built = false;
  unsigned gen = 0;  // bumped whenever arguments baked into captured graphs change
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  cudaEvent_t ev[2 * ST_COUNT] = {};
  int zchunk_phase = 0, zchunk_mom = 0;  // z planes per block of k_phase / k_mom (0: default)
  long long label_bound = 0;              // test hook: union-find loop bound (0: the cell count)
  ZsolveTc* tcz = nullptr;                // tensor-core z solve (zsolve_tc = 1)
  CUtensorMap tm_u[2], tm_v[2], tm_w[2], tm_phi[2];  // k_mom's ring boxes over U, V, W, PHI[0..1]
  int mom_tma = 1;                        // k_mom fills its interior rings by TMA (test hook: 0)
  int graph_kernels = 0;                  // kernel nodes in a captured step graph
  // 1: the inverse x transform runs fused with the projection (k_xinv_correct); 0: k_fftx_inv +
  // k_correct; -1 (the default): fused where that is the faster, nx = 512 (measured at 512^3:
  // FP64 pass pair 1.63 against 1.77 ms; at 1024^3, where k_correct streams at 96% of the copy
  // peak, and on the small boxes of the ensemble the separate passes are faster).  The fused
  // pass leaves the pressure in the spectrum only: after such a step p_lazy is set, and whatever
  // reads the pressure or reuses the spectrum first materialises it (materialise_pressure).
  int fuse_xc = -1;
  bool p_lazy = false;
  int nblk_xc = 0;                        // blocks of k_xinv_correct (partials rows)
};

// ------------------------------------------------------------------ helpers
static size_t tsize(const mhit_ctx* c) { return c->prm.poisson == MHIT_POISSON_FP64 ? 8 : 4; }
static bool refined(const mhit_ctx* c) { return c->prm.poisson == MHIT_POISSON_FP32_REFINED; }
static bool incremental(const mhit_ctx* c) { return c->prm.poisson == MHIT_POISSON_FP32_INCREMENTAL; }
// the step's inverse x transform runs inside the projection (every mode but the refinement sweep,
// whose projection reads the sum of two pressures)
static bool fused_xc(const mhit_ctx* c) {
  if (refined(c)) return false;
  return c->fuse_xc >= 0 ? c->fuse_xc != 0 : c->g.nx == 512;
}

static int check_ctx(mhit_ctx* c) {
  if (!c) return set_error(MHIT_ERR_ARG, "null context");
  cudaError_t e = cudaSetDevice(c->dev);
  if (e != cudaSuccess) return set_cuda_error(e, "cudaSetDevice", __FILE__, __LINE__);
  return MHIT_OK;
}

static std::vector<double> grid_coords(int n, double dx) {
  // x(i) = x(i-1) + dx (multi/main.f90:210-214), extended by one entry
  std::vector<double> x(n + 1, 0.0);
  double acc = 0.0;
  for (int i = 1; i <= n; ++i) {
    acc = acc + dx;
    x[i] = acc;
  }
  return x;
}

template <typename T>
static std::vector<T> twiddles(int n) {
  std::vector<T> t(2 * (size_t)n);
  const long double pi = 3.141592653589793238462643383279502884L;
  for (int m = 0; m < n; ++m) {
    const long double a = 2.0L * pi * (long double)m / (long double)n;
    t[2 * m] = (T)(double)cosl(a);
    t[2 * m + 1] = (T)(double)(-sinl(a));
  }
  return t;
}

template <typename T>
static int upload_vec(void** dst, const std::vector<T>& v) {
  MHIT_CUDA_TRY(cudaMalloc(dst, v.size() * sizeof(T)));
  MHIT_CUDA_TRY(cudaMemcpy(*dst, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice));
  return MHIT_OK;
}

static int reset_history(mhit_ctx* c, bool keep_pressure = false) {
  const size_t bytes = c->n * sizeof(double);
  MHIT_CUDA_TRY(cudaMemsetAsync(c->RU, 0, bytes, c->st));
  MHIT_CUDA_TRY(cudaMemsetAsync(c->RV, 0, bytes, c->st));
  MHIT_CUDA_TRY(cudaMemsetAsync(c->RW, 0, bytes, c->st));
  if (c->RPHI) MHIT_CUDA_TRY(cudaMemsetAsync(c->RPHI, 0, bytes, c->st));
  if (incremental(c) && !keep_pressure) {  // the pressure restarts at 0 (both predictor buffers)
    MHIT_CUDA_TRY(cudaMemsetAsync(c->P, 0, 2 * c->n * sizeof(float), c->st));
    MHIT_CUDA_TRY(cudaMemsetAsync(c->P64, 0, c->n * sizeof(double), c->st));
    c->p_lazy = false;
  }
  DevScalars s;
  memset(&s, 0, sizeof(s));
  s.gumax = 1.0;  // multi/main.f90:442
  *c->sc_host = s;
  MHIT_CUDA_TRY(cudaMemcpyAsync(c->sc, c->sc_host, sizeof(DevScalars), cudaMemcpyHostToDevice, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  c->nstep = 0;
  return MHIT_OK;
}

// Materialise the lazily removed mean into the stored velocity (before a partial overwrite).
__global__ void k_apply_mean(double* u, double* v, double* w, size_t n, DevScalars* sc) {
  const double a = sc->mean[0], b = sc->mean[1], c = sc->mean[2];
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    u[i] = u[i] - a;
    v[i] = v[i] - b;
    w[i] = w[i] - c;
  }
}

// FP32 pressure -> FP64 (exact) for a download
__global__ void k_widen(const float* __restrict__ src, double* __restrict__ dst, size_t n) {
  for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    dst[i] = (double)src[i];
}

__global__ void k_clear_mean(DevScalars* sc) {
  sc->mean[0] = 0.0;
  sc->mean[1] = 0.0;
  sc->mean[2] = 0.0;
}

// ------------------------------------------------------------------ one step
static bool stage_runs(const mhit_ctx* c, int stage, bool fz) {
  if (stage == ST_TRACER) return c->prm.partflag && c->np > 0;
  if (stage == ST_PHASE) return c->prm.phiflag != 0;
  if (stage == ST_REFINE) return c->prm.poisson == MHIT_POISSON_FP32_REFINED;
  if (stage == ST_XINV) return !fz;  // fused into the projection
  return true;
}

// Arguments of the phase and momentum stages of a step that reads buffer set `cur`.
static PhaseArgs phase_args(const mhit_ctx* c, double alpha, double beta, int cur) {
  const int nxt = cur ^ 1;
  PhaseArgs a;
  a.g = c->g;
  a.phi = c->PHI[cur];
  a.u = c->U[cur];
  a.v = c->V[cur];
  a.w = c->W[cur];
  a.phin = c->PHI[nxt];
  a.rphio = c->RPHI;
  a.sc = c->sc;
  a.alpha = alpha;
  a.beta = beta;
  a.clamp = c->prm.acdi_clamp;
  a.zchunk = c->zchunk_phase;
  return a;
}

static MomArgs mom_args(const mhit_ctx* c, double alpha, double beta, int cur) {
  const int nxt = cur ^ 1;
  MomArgs a;
  a.g = c->g;
  a.u = c->U[cur];
  a.v = c->V[cur];
  a.w = c->W[cur];
  a.un = c->U[nxt];
  a.vn = c->V[nxt];
  a.wn = c->W[nxt];
  a.ru = c->RU;
  a.rv = c->RV;
  a.rw = c->RW;
  a.phi = c->prm.phiflag ? c->PHI[nxt] : nullptr;
  a.tabs = c->tabs;
  a.sc = c->sc;
  a.alpha = alpha;
  a.beta = beta;
  a.zchunk = c->zchunk_mom;
  a.tma = c->mom_tma;
  a.tmu = c->tm_u[cur];
  a.tmv = c->tm_v[cur];
  a.tmw = c->tm_w[cur];
  if (c->prm.phiflag) a.tmphi = c->tm_phi[nxt];
  return a;
}

// Launch one stage of the step that reads buffer set `cur` and writes set `cur ^ 1`; fz: the
// inverse x transform runs inside the projection stage.
static int enqueue_stage(mhit_ctx* c, int stage, double alpha, double beta, int cur, bool fz) {
  const int nxt = cur ^ 1;
  const mhit_params& p = c->prm;
  if (!stage_runs(c, stage, fz)) return MHIT_OK;
  switch (stage) {
    case ST_TRACER: {
      TracerArgs a;
      a.g = c->g;
      a.part = c->part;
      a.np = c->np;
      a.npmax = c->np;
      a.u = c->U[cur];
      a.v = c->V[cur];
      a.w = c->W[cur];
      a.sc = c->sc;
      a.alpha = alpha;
      a.beta = beta;
      a.lx = 8.0 * atan(1.0);
      a.interp = p.interp;
      a.yz_shift = p.yz_shift;
      MHIT_CUDA_TRY(launch_tracer(a, c->st));
      return MHIT_OK;
    }
    case ST_PHASE: {
      MHIT_CUDA_TRY(launch_phase(phase_args(c, alpha, beta, cur), c->st));
      return MHIT_OK;
    }
    case ST_MOM: {
      MHIT_CUDA_TRY(launch_mom(mom_args(c, alpha, beta, cur), c->st));
      return MHIT_OK;
    }
    case ST_XFWD:
    case ST_YFWD:
    case ST_ZSOLVE:
    case ST_YINV:
    case ST_XINV:
    case ST_REFINE: {
      PoissonArgs a;
      a.g = c->g;
      a.fp32 = p.poisson != MHIT_POISSON_FP64;
      a.u = c->U[nxt];
      a.v = c->V[nxt];
      a.w = c->W[nxt];
      a.spec = c->spec;
      a.p = c->P;
      a.twx = c->twx;
      a.twy = c->twy;
      a.twz = c->twz;
      a.k2x = c->k2x;
      a.k2y = c->k2y;
      a.k2z = c->k2z;
      a.cdiv = p.rho * c->g.dxi / p.dt;  // (rho*dxi/dt), multi/main.f90:841
      a.ntot = (double)c->g.nx * (double)c->g.ny * (double)c->g.nz;
      a.tcz = c->tcz;
      a.sc = c->sc;
      if (incremental(c)) {
        // the residual of the predictor Q[cur] in the x pass; the x-inverse writes the pressure
        // Q[cur] + delta to P64 in FP64 and its FP32 rounding to Q[nxt]
        if (stage == ST_XFWD) a.presid = c->Q[cur];
        if (stage == ST_XINV) {
          a.qin = c->Q[cur];
          a.qout = c->Q[nxt];
          a.p64 = c->P64;
        }
      }
      if (stage != ST_REFINE) {
        MHIT_CUDA_TRY(poisson_stage(a, stage - ST_XFWD, c->st));
        return MHIT_OK;
      }
      // one FP64 residual sweep: the x pass forms r = rhs - L_h P in FP64, L_h delta = r in FP32
      // (delta -> P2); the projection reads p = P + P2
      a.presid = static_cast<const float*>(c->P);
      a.p = c->P2;
      for (int s = 0; s < PSTAGE_COUNT; ++s) MHIT_CUDA_TRY(poisson_stage(a, s, c->st));
      return MHIT_OK;
    }
    case ST_CORRECT: {
      if (fz) {
        XcArgs x;
        x.g = c->g;
        x.fp32 = p.poisson != MHIT_POISSON_FP64;
        x.spec = c->spec;
        x.twx = c->twx;
        x.u = c->U[nxt];
        x.v = c->V[nxt];
        x.w = c->W[nxt];
        if (incremental(c)) {
          x.qold = c->Q[cur];
          x.qnew = c->Q[nxt];
        }
        x.partials = c->partials;
        x.sc = c->sc;
        MHIT_CUDA_TRY(launch_xinv_correct(x, c->st));
        return MHIT_OK;
      }
      CorrectArgs a;
      a.g = c->g;
      a.u = c->U[nxt];
      a.v = c->V[nxt];
      a.w = c->W[nxt];
      a.p = incremental(c) ? static_cast<void*>(c->P64) : c->P;
      a.fp32 = p.poisson != MHIT_POISSON_FP64 && !incremental(c);
      a.pd = refined(c) ? c->P2 : nullptr;
      a.partials = c->partials;
      a.nblocks = c->nblk;
      a.sc = c->sc;
      MHIT_CUDA_TRY(launch_correct(a, c->st));
      return MHIT_OK;
    }
  }
  return set_error(MHIT_ERR_ARG, "unknown stage");
}

static int enqueue_step(mhit_ctx* c, double alpha, double beta, int cur, bool profile) {
  const bool fz = fused_xc(c);
  for (int s = 0; s < ST_COUNT; ++s) {
    const bool ran = stage_runs(c, s, fz);
    if (profile && ran) MHIT_CUDA_TRY(cudaEventRecord(c->ev[2 * s], c->st));
    int rc = enqueue_stage(c, s, alpha, beta, cur, fz);
    if (rc) return rc;
    if (profile && ran) MHIT_CUDA_TRY(cudaEventRecord(c->ev[2 * s + 1], c->st));
  }
  return MHIT_OK;
}

// The pressure of the last step into P (P64 in the incremental solve) when the fused projection
// left it in the spectrum: the inverse x transform of the y-inverted spectrum, which no kernel
// touches between steps until this runs; in the incremental solve added to the predictor that
// step read, Q[cur ^ 1] (the one it wrote, Q[cur], already holds fl32 of the sum).
static int materialise_pressure(mhit_ctx* c) {
  if (!c->p_lazy) return MHIT_OK;
  PoissonArgs a;
  a.g = c->g;
  a.fp32 = c->prm.poisson != MHIT_POISSON_FP64;
  a.u = a.v = a.w = nullptr;
  a.spec = c->spec;
  a.p = c->P;
  a.twx = c->twx;
  a.twy = c->twy;
  a.twz = c->twz;
  a.k2x = a.k2y = a.k2z = nullptr;
  a.cdiv = 0.0;
  a.ntot = (double)c->n;
  if (incremental(c)) {
    a.qin = c->Q[c->cur ^ 1];
    a.qout = nullptr;
    a.p64 = c->P64;
  }
  MHIT_CUDA_TRY(poisson_stage(a, PSTAGE_XINV, c->st));
  c->p_lazy = false;
  return MHIT_OK;
}

static int build_graphs(mhit_ctx* c) {
  for (int par = 0; par < 2; ++par) {
    cudaGraph_t graph;
    MHIT_CUDA_TRY(cudaStreamBeginCapture(c->st, cudaStreamCaptureModeThreadLocal));
    int rc = enqueue_step(c, 1.5, 0.5, par, false);
    cudaError_t e = cudaStreamEndCapture(c->st, &graph);
    if (rc) return rc;
    if (e != cudaSuccess) return set_cuda_error(e, "cudaStreamEndCapture", __FILE__, __LINE__);
    // count the kernels one replayed step launches (reported by mhit_kernels_per_step)
    size_t nn = 0;
    e = cudaGraphGetNodes(graph, nullptr, &nn);
    std::vector<cudaGraphNode_t> nodes(nn);
    if (e == cudaSuccess && nn) e = cudaGraphGetNodes(graph, nodes.data(), &nn);
    int nk = 0;
    for (size_t q = 0; e == cudaSuccess && q < nn; ++q) {
      cudaGraphNodeType t;
      e = cudaGraphNodeGetType(nodes[q], &t);
      if (e == cudaSuccess && t == cudaGraphNodeTypeKernel) ++nk;
    }
    if (e != cudaSuccess) {
      cudaGraphDestroy(graph);
      return set_cuda_error(e, "cudaGraphGetNodes", __FILE__, __LINE__);
    }
    c->graph_kernels = nk;
    e = cudaGraphInstantiate(&c->gexec[par], graph, 0);
    cudaGraphDestroy(graph);
    if (e != cudaSuccess) return set_cuda_error(e, "cudaGraphInstantiate", __FILE__, __LINE__);
  }
  c->graph_built = true;
  return MHIT_OK;
}

// enqueue nsteps without the final flag check
static int enqueue_steps(mhit_ctx* c, int nsteps) {
  for (int s = 0; s < nsteps; ++s) {
    int rc;
    if (c->nstep == 0) {
      rc = enqueue_step(c, 1.0, 0.0, c->cur, false);  // Euler first step, multi/main.f90:440-441
    } else if (c->prm.use_graph) {
      if (!c->graph_built && (rc = build_graphs(c))) return rc;
      MHIT_CUDA_TRY(cudaGraphLaunch(c->gexec[c->cur], c->st));
      rc = MHIT_OK;
    } else {
      rc = enqueue_step(c, 1.5, 0.5, c->cur, false);  // AB2, multi/main.f90:801-802
    }
    if (rc) return rc;
    c->cur ^= 1;
    c->nstep++;
    c->p_lazy = fused_xc(c);
  }
  return MHIT_OK;
}

static int fetch_scalars(mhit_ctx* c) {
  MHIT_CUDA_TRY(cudaMemcpyAsync(c->sc_host, c->sc, sizeof(DevScalars), cudaMemcpyDeviceToHost, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return MHIT_OK;
}

// ------------------------------------------------------------------ C ABI
extern "C" {

int mhit_abi_version(void) { return MHIT_ABI_VERSION; }

const char* mhit_last_error(void) { return g_err.c_str(); }

int mhit_params_default(mhit_params* p) {
  if (!p) return set_error(MHIT_ERR_ARG, "null params");
  memset(p, 0, sizeof(*p));
  p->nx = p->ny = p->nz = 64;
  // multi/input.inp:7-16
  p->dt = 0.0002;
  p->mu = 0.006;
  p->rho = 1.0;
  p->f1 = p->f2 = p->f3 = 1.0;
  p->k0 = 2.0;
  p->radius = 0.5;
  p->sigma = 1.0;
  p->epsr = 1.0;
  p->npart = 0;
  p->poisson = MHIT_POISSON_FP64;
  p->laplacian = MHIT_LAP_EXACT;
  p->interp = MHIT_INTERP_LINEAR1D;
  p->yz_shift = 1;
  p->use_graph = 1;
  p->device = 0;
  return MHIT_OK;
}

static int parse_num(FILE* f, double* out, int lineno, const char* path) {
  char line[512];
  if (!fgets(line, sizeof(line), f)) {
    char b[600];
    snprintf(b, sizeof(b), "%s: missing line %d", path, lineno);
    return set_error(MHIT_ERR_IO, b);
  }
  // first token; Fortran d/D exponent -> e
  char tok[128];
  if (sscanf(line, "%127s", tok) != 1) {
    char b[600];
    snprintf(b, sizeof(b), "%s: empty line %d", path, lineno);
    return set_error(MHIT_ERR_IO, b);
  }
  for (char* q = tok; *q; ++q)
    if (*q == 'd' || *q == 'D') *q = 'e';
  char* end = nullptr;
  *out = strtod(tok, &end);
  if (end == tok) {
    char b[600];
    snprintf(b, sizeof(b), "%s: line %d is not a number: %s", path, lineno, tok);
    return set_error(MHIT_ERR_IO, b);
  }
  return MHIT_OK;
}

int mhit_read_input(const char* path, mhit_params* p, mhit_run* run) {
  if (!path || !p) return set_error(MHIT_ERR_ARG, "null argument");
  FILE* f = fopen(path, "r");
  if (!f) return set_error(MHIT_ERR_IO, std::string("cannot open ") + path);
  double v[18];
  for (int i = 0; i < 18; ++i) {
    int rc = parse_num(f, &v[i], i + 1, path);
    if (rc) {
      fclose(f);
      return rc;
    }
  }
  fclose(f);
  // multi/readinput.f90:14-35, in file order
  if (run) {
    run->restart = (int)v[0];
    run->tstart = (int)v[1];
    run->tfin = (int)v[2];
    run->dump = (int)v[3];
    run->inflow = (int)v[4];
    run->inphi = (int)v[5];
    run->inpart = (int)v[17];
  }
  p->dt = v[6];
  p->mu = v[7];
  p->rho = v[8];
  p->f1 = v[9];
  p->f2 = v[10];
  p->f3 = v[11];
  p->k0 = v[12];
  p->radius = v[13];
  p->sigma = v[14];
  p->epsr = v[15];
  p->npart = (int)v[16];
  return MHIT_OK;
}

void mhit_destroy(mhit_ctx* c) {
  if (!c) return;
  cudaSetDevice(c->dev);
  if (c->st) cudaStreamSynchronize(c->st);
  for (int i = 0; i < 2; ++i) {
    if (c->gexec[i]) cudaGraphExecDestroy(c->gexec[i]);
    cudaFree(c->U[i]);
    cudaFree(c->V[i]);
    cudaFree(c->W[i]);
    cudaFree(c->PHI[i]);
  }
  cudaFree(c->RU);
  cudaFree(c->RV);
  cudaFree(c->RW);
  cudaFree(c->RPHI);
  cudaFree(c->P);
  cudaFree(c->P2);
  cudaFree(c->P64);
  cudaFree(c->Pw);
  cudaFree(c->lab_small);
  cudaFree(c->lab_acc);
  cudaFree(c->spec);
  cudaFree(c->spec64);
  for (void* t : c->tw64) cudaFree(t);
  cudaFree(c->twx);
  cudaFree(c->twy);
  cudaFree(c->twz);
  cudaFree(c->k2x);
  cudaFree(c->k2y);
  cudaFree(c->k2z);
  cudaFree(c->tabs);
  cudaFree(c->partials);
  zsolve_tc_destroy(c->tcz);
  cudaFree(c->sc);
  cudaFree(c->part);
  if (c->sc_host) cudaFreeHost(c->sc_host);
  for (int i = 0; i < 2 * ST_COUNT; ++i)
    if (c->ev[i]) cudaEventDestroy(c->ev[i]);
  if (c->st) cudaStreamDestroy(c->st);
  delete c;
}

static int init_impl(const mhit_params* p, mhit_ctx* c) {
  c->prm = *p;
  c->dev = p->device;
  MHIT_CUDA_TRY(cudaSetDevice(c->dev));
  MHIT_CUDA_TRY(cudaStreamCreateWithFlags(&c->st, cudaStreamNonBlocking));
  for (int i = 0; i < 2 * ST_COUNT; ++i) MHIT_CUDA_TRY(cudaEventCreate(&c->ev[i]));
  Geo& g = c->g;
  g.nx = p->nx;
  g.ny = p->ny;
  g.nz = p->nz;
  g.nkx = p->nx / 2 + 1;
  g.pitch = (g.nkx + 15) / 16 * 16;
  // multi/readinput.f90:114-124
  const double twopi = 8.0 * atan(1.0);
  const double lx = twopi;
  g.dx = lx / p->nx;
  g.dxi = 1.0 / g.dx;
  g.ddxi = 1.0 / g.dx / g.dx;
  g.rhoi = 1.0 / p->rho;
  g.eps = p->epsr * g.dx;
  g.epsi = 1.0 / g.eps;
  g.dt = p->dt;
  g.mu = p->mu;
  g.rho = p->rho;
  g.sigma = p->sigma;
  g.f1 = p->f1;
  g.f2 = p->f2;
  g.f3 = p->f3;
  const size_t n = (size_t)g.nx * g.ny * g.nz;
  c->n = n;
  const size_t fb = n * sizeof(double);
  int rc0;
  for (int i = 0; i < 2; ++i) {
    MHIT_CUDA_TRY(cudaMalloc(&c->U[i], fb));
    MHIT_CUDA_TRY(cudaMalloc(&c->V[i], fb));
    MHIT_CUDA_TRY(cudaMalloc(&c->W[i], fb));
    MHIT_CUDA_TRY(cudaMemset(c->U[i], 0, fb));
    MHIT_CUDA_TRY(cudaMemset(c->V[i], 0, fb));
    MHIT_CUDA_TRY(cudaMemset(c->W[i], 0, fb));
    if (p->phiflag) {
      MHIT_CUDA_TRY(cudaMalloc(&c->PHI[i], fb));
      MHIT_CUDA_TRY(cudaMemset(c->PHI[i], 0, fb));
    }
  }
  for (int i = 0; i < 2; ++i) {  // the momentum kernel's TMA boxes over each ping-pong buffer
    if ((rc0 = mom_field_map(&c->tm_u[i], c->U[i], g.nx, g.ny, g.nz, false))) return rc0;
    if ((rc0 = mom_field_map(&c->tm_v[i], c->V[i], g.nx, g.ny, g.nz, false))) return rc0;
    if ((rc0 = mom_field_map(&c->tm_w[i], c->W[i], g.nx, g.ny, g.nz, false))) return rc0;
    if (p->phiflag && (rc0 = mom_field_map(&c->tm_phi[i], c->PHI[i], g.nx, g.ny, g.nz, true))) return rc0;
  }
  MHIT_CUDA_TRY(cudaMalloc(&c->RU, fb));
  MHIT_CUDA_TRY(cudaMalloc(&c->RV, fb));
  MHIT_CUDA_TRY(cudaMalloc(&c->RW, fb));
  if (p->phiflag) MHIT_CUDA_TRY(cudaMalloc(&c->RPHI, fb));
  const size_t ts = tsize(c);
  // the incremental solve keeps two FP32 predictors (read one, write the other), in one block
  MHIT_CUDA_TRY(cudaMalloc(&c->P, (incremental(c) ? 2 : 1) * n * ts));
  if (incremental(c)) {
    c->Q[0] = static_cast<float*>(c->P);
    c->Q[1] = c->Q[0] + n;
  }
  if (refined(c)) {
    MHIT_CUDA_TRY(cudaMalloc(&c->P2, n * sizeof(float)));
    MHIT_CUDA_TRY(cudaMemset(c->P2, 0, n * sizeof(float)));
  }
  if (refined(c) || incremental(c)) {
    MHIT_CUDA_TRY(cudaMalloc(&c->P64, n * sizeof(double)));
    MHIT_CUDA_TRY(cudaMemset(c->P64, 0, n * sizeof(double)));
  }
  MHIT_CUDA_TRY(cudaMemset(c->P, 0, (incremental(c) ? 2 : 1) * n * ts));
  MHIT_CUDA_TRY(cudaMalloc(&c->spec, (size_t)g.pitch * g.ny * g.nz * 2 * ts));
  MHIT_CUDA_TRY(cudaMemset(c->spec, 0, (size_t)g.pitch * g.ny * g.nz * 2 * ts));
  int rc;
  if (p->zsolve_tc && (rc = zsolve_tc_create(g, c->spec, &c->tcz))) return rc;
  if (ts == 4) {
    if ((rc = upload_vec(&c->twx, twiddles<float>(g.nx)))) return rc;
    if ((rc = upload_vec(&c->twy, twiddles<float>(g.ny)))) return rc;
    if ((rc = upload_vec(&c->twz, twiddles<float>(g.nz)))) return rc;
  } else {
    if ((rc = upload_vec(&c->twx, twiddles<double>(g.nx)))) return rc;
    if ((rc = upload_vec(&c->twy, twiddles<double>(g.ny)))) return rc;
    if ((rc = upload_vec(&c->twz, twiddles<double>(g.nz)))) return rc;
  }
  // k^2 per axis (multi/main.f90:234-240, 889), or the modified wavenumber.  The cells are cubes
  // of side dx = lx/nx, so an axis of nn cells is nn dx long: its wavenumber of index kk is
  // kk nx/nn (in units of 2 pi/lx = 1) and its modified symbol (2 - 2 cos(kk 2 pi/nn))/dx^2.  On
  // the reference's cubic box these are the integer kk and (2 - 2 cos(kk dx))/dx^2.
  auto k2tab = [&](int nn, int len) {
    std::vector<double> t(len);
    const double h = lx / nn, scale = (double)p->nx / (double)nn;
    for (int i = 0; i < len; ++i) {
      const double kk = (i < nn / 2) ? (double)i : (double)(i - nn);
      const double kp = kk * scale;
      t[i] = p->laplacian == MHIT_LAP_MODIFIED ? (2.0 - 2.0 * cos(kk * h)) * g.ddxi : kp * kp;
    }
    return t;
  };
  if ((rc = upload_vec((void**)&c->k2x, k2tab(g.nx, g.nkx)))) return rc;
  if ((rc = upload_vec((void**)&c->k2y, k2tab(g.ny, g.ny)))) return rc;
  if ((rc = upload_vec((void**)&c->k2z, k2tab(g.nz, g.nz)))) return rc;
  // forcing tables (multi/main.f90:244-250; y/z read one entry on, see header)
  {
    std::vector<double> t;
    const int ns[3] = {g.nx, g.ny, g.nz};
    std::vector<double> sv[3], cv[3];
    for (int ax = 0; ax < 3; ++ax) {
      const int nn = ns[ax];
      std::vector<double> xc = grid_coords(nn, g.dx);
      const int off = ax == 0 ? 0 : p->yz_shift;
      for (int i = 0; i < nn; ++i) {
        t.push_back(sin(p->k0 * xc[i + off] + g.dx / 2));
      }
      for (int i = 0; i < nn; ++i) {
        t.push_back(cos(p->k0 * xc[i + off] + g.dx / 2));
      }
    }
    if ((rc = upload_vec((void**)&c->tabs, t))) return rc;
  }
  c->nblk = correct_blocks(g);
  c->nblk_xc = xc_blocks(g, 0);
  MHIT_CUDA_TRY(cudaMalloc(&c->partials, (size_t)std::max(c->nblk, c->nblk_xc) * 6 * sizeof(double)));
  MHIT_CUDA_TRY(cudaMalloc(&c->sc, sizeof(DevScalars)));
  MHIT_CUDA_TRY(cudaMallocHost(&c->sc_host, sizeof(DevScalars)));
  return reset_history(c);
}

int mhit_init(const mhit_params* p, mhit_ctx** out) {
  if (!p || !out) return set_error(MHIT_ERR_ARG, "null argument");
  *out = nullptr;
  if (!poisson_size_supported(p->nx, true) || !poisson_size_supported(p->ny, false) ||
      !poisson_size_supported(p->nz, false) || p->nx < 16) {
    char b[256];
    snprintf(b, sizeof(b), "unsupported grid %dx%dx%d (each of 16,32,64,128,192,256,512,1024; nx even)", p->nx, p->ny,
             p->nz);
    return set_error(MHIT_ERR_ARG, b);
  }
  if (p->nx != 2 * (p->nx / 2) || !(p->dt > 0) || !(p->rho > 0) || !(p->epsr > 0))
    return set_error(MHIT_ERR_ARG, "dt, rho and epsr must be positive");
  if (p->poisson != MHIT_POISSON_FP64 && p->poisson != MHIT_POISSON_FP32 && p->poisson != MHIT_POISSON_FP32_REFINED &&
      p->poisson != MHIT_POISSON_FP32_INCREMENTAL)
    return set_error(MHIT_ERR_ARG, "poisson must be MHIT_POISSON_FP64, _FP32, _FP32_REFINED or _FP32_INCREMENTAL");
  if ((p->poisson == MHIT_POISSON_FP32_REFINED || p->poisson == MHIT_POISSON_FP32_INCREMENTAL) &&
      p->laplacian != MHIT_LAP_MODIFIED)
    return set_error(MHIT_ERR_ARG, "MHIT_POISSON_FP32_REFINED and _FP32_INCREMENTAL need laplacian = MHIT_LAP_MODIFIED "
                                   "(their residual is the 7-point operator)");
  if (p->laplacian != MHIT_LAP_EXACT && p->laplacian != MHIT_LAP_MODIFIED)
    return set_error(MHIT_ERR_ARG, "laplacian must be MHIT_LAP_EXACT or MHIT_LAP_MODIFIED");
  if (p->interp != MHIT_INTERP_LINEAR1D && p->interp != MHIT_INTERP_TRILINEAR)
    return set_error(MHIT_ERR_ARG, "interp must be MHIT_INTERP_LINEAR1D or MHIT_INTERP_TRILINEAR");
  if (p->yz_shift != 0 && p->yz_shift != 1) return set_error(MHIT_ERR_ARG, "yz_shift must be 0 or 1");
  if (p->acdi_clamp != 0 && p->acdi_clamp != 1) return set_error(MHIT_ERR_ARG, "acdi_clamp must be 0 or 1");
  if (p->zsolve_tc != 0 && p->zsolve_tc != 1) return set_error(MHIT_ERR_ARG, "zsolve_tc must be 0 or 1");
  if (p->zsolve_tc && (p->poisson == MHIT_POISSON_FP64 || p->nz != 512))
    return set_error(MHIT_ERR_ARG, "zsolve_tc needs nz = 512 and a FP32 Poisson mode");
  int ndev = 0;
  cudaError_t e = cudaGetDeviceCount(&ndev);
  if (e != cudaSuccess) return set_cuda_error(e, "cudaGetDeviceCount", __FILE__, __LINE__);
  if (p->device < 0 || p->device >= ndev) return set_error(MHIT_ERR_ARG, "device ordinal out of range");
  mhit_ctx* c = new mhit_ctx();
  int rc = init_impl(p, c);
  if (rc) {
    std::string keep = g_err;
    mhit_destroy(c);
    g_err = keep;
    return rc;
  }
  *out = c;
  return MHIT_OK;
}

int mhit_upload_fields(mhit_ctx* c, const double* u, const double* v, const double* w, const double* phi) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!u || !v || !w) return set_error(MHIT_ERR_ARG, "u, v and w are required");
  if (c->prm.phiflag && !phi) return set_error(MHIT_ERR_ARG, "phi is required when phiflag=1");
  const size_t fb = c->n * sizeof(double);
  c->cur = 0;
  MHIT_CUDA_TRY(cudaMemcpyAsync(c->U[0], u, fb, cudaMemcpyHostToDevice, c->st));
  MHIT_CUDA_TRY(cudaMemcpyAsync(c->V[0], v, fb, cudaMemcpyHostToDevice, c->st));
  MHIT_CUDA_TRY(cudaMemcpyAsync(c->W[0], w, fb, cudaMemcpyHostToDevice, c->st));
  if (c->prm.phiflag) MHIT_CUDA_TRY(cudaMemcpyAsync(c->PHI[0], phi, fb, cudaMemcpyHostToDevice, c->st));
  return reset_history(c);
}

// Replace the tracer table by an allocated, unfilled one of npart rows (none for 0).
static int reset_particles(mhit_ctx* c, int npart) {
  if (c->part) {
    MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
    cudaFree(c->part);
    c->part = nullptr;
  }
  c->np = npart;
  c->gen++;
  // the tracer kernel's pointer (and whether it runs at all) is baked into captured graphs
  for (int i = 0; i < 2; ++i)
    if (c->gexec[i]) {
      cudaGraphExecDestroy(c->gexec[i]);
      c->gexec[i] = nullptr;
    }
  c->graph_built = false;
  if (npart > 0) MHIT_CUDA_TRY(cudaMalloc(&c->part, (size_t)npart * 12 * sizeof(double)));
  return MHIT_OK;
}

int mhit_upload_particles(mhit_ctx* c, const double* part, int npart) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!c->prm.partflag) return set_error(MHIT_ERR_STATE, "context was created with partflag=0");
  if (npart < 0 || (npart > 0 && !part)) return set_error(MHIT_ERR_ARG, "bad particle table");
  if ((rc = reset_particles(c, npart))) return rc;
  if (npart == 0) return MHIT_OK;
  MHIT_CUDA_TRY(cudaMemcpyAsync(c->part, part, (size_t)npart * 12 * sizeof(double), cudaMemcpyHostToDevice, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return MHIT_OK;
}

int mhit_init_particles(mhit_ctx* c, int npart, unsigned long long seed) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!c->prm.partflag) return set_error(MHIT_ERR_STATE, "context was created with partflag=0");
  if (npart < 1) return set_error(MHIT_ERR_ARG, "npart must be positive");
  if ((rc = reset_particles(c, npart))) return rc;
  const double lx = 8.0 * std::atan(1.0);
  MHIT_CUDA_TRY(launch_init_particles(c->part, npart, seed, lx, c->prm.ny == c->prm.nx ? lx : c->g.dx * c->prm.ny,
                                      c->prm.nz == c->prm.nx ? lx : c->g.dx * c->prm.nz, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return MHIT_OK;
}

int mhit_download_particles(mhit_ctx* c, double* part, int npart) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (npart != c->np) return set_error(MHIT_ERR_ARG, "npart does not match the uploaded table");
  if (npart == 0) return MHIT_OK;
  if (!part) return set_error(MHIT_ERR_ARG, "null particle buffer");
  MHIT_CUDA_TRY(cudaMemcpyAsync(part, c->part, (size_t)npart * 12 * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return MHIT_OK;
}

int mhit_step(mhit_ctx* c, int nsteps) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (nsteps < 0) return set_error(MHIT_ERR_ARG, "nsteps < 0");
  if ((rc = enqueue_steps(c, nsteps))) return rc;
  if ((rc = fetch_scalars(c))) return rc;
  if (c->sc_host->flag & 4)
    return set_error(MHIT_ERR_TIMEOUT, "the tensor-core z solve gave up on a bounded wait (results invalid)");
  if (c->sc_host->flag & 1) return set_error(MHIT_ERR_NAN, "NaN in the velocity field");
  if (c->sc_host->flag & 2) {
    char b[128];
    snprintf(b, sizeof(b), "CFL %.6g > 7 (multi/main.f90:1006 stops here)", c->sc_host->cfl);
    return set_error(MHIT_ERR_CFL, b);
  }
  return MHIT_OK;
}

int mhit_time_steps(mhit_ctx* c, int nsteps, double* ms) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!ms || nsteps < 0) return set_error(MHIT_ERR_ARG, "bad argument");
  MHIT_CUDA_TRY(cudaEventRecord(c->ev[0], c->st));
  if ((rc = enqueue_steps(c, nsteps))) return rc;
  MHIT_CUDA_TRY(cudaEventRecord(c->ev[1], c->st));
  MHIT_CUDA_TRY(cudaEventSynchronize(c->ev[1]));
  float f = 0.f;
  MHIT_CUDA_TRY(cudaEventElapsedTime(&f, c->ev[0], c->ev[1]));
  *ms = f;
  return MHIT_OK;
}

int mhit_kernels_per_step(mhit_ctx* c, int* n) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!n) return set_error(MHIT_ERR_ARG, "null argument");
  if (!c->graph_built && (rc = build_graphs(c))) return rc;
  *n = c->graph_kernels;
  return MHIT_OK;
}

int mhit_profile_step(mhit_ctx* c, double* ms, const char** names, int* nstages) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!ms || !nstages || *nstages < ST_COUNT) return set_error(MHIT_ERR_ARG, "need room for all stages");
  const bool first = c->nstep == 0;
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  if ((rc = materialise_pressure(c))) return rc;  // not needed by the step; keeps the flag exact
  // mark stages that do not run
  for (int i = 0; i < ST_COUNT; ++i) ms[i] = -1.0;
  if ((rc = enqueue_step(c, first ? 1.0 : 1.5, first ? 0.0 : 0.5, c->cur, true))) return rc;
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  const bool fz = fused_xc(c);
  for (int i = 0; i < ST_COUNT; ++i) {
    if (stage_runs(c, i, fz)) {
      float f = 0.f;
      MHIT_CUDA_TRY(cudaEventElapsedTime(&f, c->ev[2 * i], c->ev[2 * i + 1]));
      ms[i] = f;
    }
    if (names) names[i] = (i == ST_CORRECT && fz) ? kFusedCorrectName : kStageNames[i];
  }
  *nstages = ST_COUNT;
  c->cur ^= 1;
  c->nstep++;
  c->p_lazy = fz;
  return MHIT_OK;
}

int mhit_download_fields(mhit_ctx* c, double* u, double* v, double* w, double* p, double* phi) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (phi && !c->prm.phiflag) return set_error(MHIT_ERR_STATE, "context was created with phiflag=0");
  const size_t n = c->n, fb = n * sizeof(double);
  double* outs[3] = {u, v, w};
  double* srcs[3] = {c->U[c->cur], c->V[c->cur], c->W[c->cur]};
  if (u || v || w) {
    // the lazily removed mean (multi/main.f90:977-981) is made explicit on the device: the
    // stored value minus the mean, the same double every reader computes, so later steps are
    // unchanged
    k_apply_mean<<<148 * 4, 256, 0, c->st>>>(c->U[c->cur], c->V[c->cur], c->W[c->cur], n, c->sc);
    MHIT_CUDA_TRY(cudaGetLastError());
    k_clear_mean<<<1, 1, 0, c->st>>>(c->sc);
    MHIT_CUDA_TRY(cudaGetLastError());
  }
  for (int q = 0; q < 3; ++q) {
    if (!outs[q]) continue;
    MHIT_CUDA_TRY(cudaMemcpyAsync(outs[q], srcs[q], fb, cudaMemcpyDeviceToHost, c->st));
  }
  if (phi) MHIT_CUDA_TRY(cudaMemcpyAsync(phi, c->PHI[c->cur], fb, cudaMemcpyDeviceToHost, c->st));
  if (p) {
    if ((rc = materialise_pressure(c))) return rc;
    const double* src = static_cast<const double*>(c->P);
    if (incremental(c)) {  // the FP64 pressure of the last projection
      src = c->P64;
    } else if (c->P2) {  // refinement: materialise p = P + P2 in FP64
      MHIT_CUDA_TRY(launch_combine(static_cast<const float*>(c->P), c->P2, c->P64, c->n, c->st));
      src = c->P64;
    } else if (tsize(c) == 4) {
      if (!c->Pw) MHIT_CUDA_TRY(cudaMalloc(&c->Pw, fb));
      k_widen<<<148 * 4, 256, 0, c->st>>>(static_cast<const float*>(c->P), c->Pw, n);
      MHIT_CUDA_TRY(cudaGetLastError());
      src = c->Pw;
    }
    MHIT_CUDA_TRY(cudaMemcpyAsync(p, src, fb, cudaMemcpyDeviceToHost, c->st));
  }
  return fetch_scalars(c);  // synchronises the stream: the copies are complete
}

int mhit_diagnostics(mhit_ctx* c, mhit_diag* d) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!d) return set_error(MHIT_ERR_ARG, "null diag");
  // the partials buffer of the projection is reused (stream ordered)
  DiagArgs a;
  a.g = c->g;
  a.u = c->U[c->cur];
  a.v = c->V[c->cur];
  a.w = c->W[c->cur];
  a.partials = c->partials;
  a.nblocks = c->nblk;
  a.sc = c->sc;
  a.nu = c->prm.mu / c->prm.rho;
  a.dxd = c->g.dx;
  MHIT_CUDA_TRY(launch_diag(a, c->st));
  if ((rc = fetch_scalars(c))) return rc;
  const DevScalars& s = *c->sc_host;
  d->nstep = c->nstep;
  d->gumax = s.gumax;
  d->cfl = s.cfl;
  for (int q = 0; q < 3; ++q) d->mean[q] = s.mean[q];
  d->maxdiv = s.diag[0];
  d->ke = s.diag[1];
  d->dissipation = s.diag[2];
  d->flags = s.flag;
  return MHIT_OK;
}

static const char* kFieldNames[6] = {"", "u", "v", "w", "p", "phi"};

int mhit_write_field(mhit_ctx* c, const char* dir, int t, int fieldn) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!dir || fieldn < 1 || fieldn > 5) return set_error(MHIT_ERR_ARG, "fieldn must be 1..5");
  if (fieldn == 5 && !c->prm.phiflag) return set_error(MHIT_ERR_STATE, "context was created with phiflag=0");
  std::vector<double> buf(c->n);
  double* ptrs[6] = {nullptr, nullptr, nullptr, nullptr, nullptr, nullptr};
  ptrs[fieldn] = buf.data();
  if ((rc = mhit_download_fields(c, ptrs[1], ptrs[2], ptrs[3], ptrs[4], ptrs[5]))) return rc;
  char path[4096];
  // './output/u_',t,'.dat' with i8.8 (multi/readwrite.f90:41)
  snprintf(path, sizeof(path), "%s/%s_%08d.dat", dir, kFieldNames[fieldn], t);
  FILE* f = fopen(path, "wb");
  if (!f) return set_error(MHIT_ERR_IO, std::string("cannot create ") + path);
  const size_t wr = fwrite(buf.data(), sizeof(double), c->n, f);
  const int cl = fclose(f);
  if (wr != c->n || cl != 0) return set_error(MHIT_ERR_IO, std::string("short write to ") + path);
  return MHIT_OK;
}

int mhit_read_field(mhit_ctx* c, const char* path, int fieldn) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!path || fieldn < 1 || fieldn > 5) return set_error(MHIT_ERR_ARG, "fieldn must be 1..5");
  if (fieldn == 5 && !c->prm.phiflag) return set_error(MHIT_ERR_STATE, "context was created with phiflag=0");
  std::vector<double> buf(c->n);
  FILE* f = fopen(path, "rb");
  if (!f) return set_error(MHIT_ERR_IO, std::string("cannot open ") + path);
  const size_t rd = fread(buf.data(), sizeof(double), c->n, f);
  fclose(f);
  if (rd != c->n) return set_error(MHIT_ERR_IO, std::string("short read from ") + path);
  const size_t fb = c->n * sizeof(double);
  // make the stored velocity explicit before replacing one component
  k_apply_mean<<<148 * 4, 256, 0, c->st>>>(c->U[c->cur], c->V[c->cur], c->W[c->cur], c->n, c->sc);
  MHIT_CUDA_TRY(cudaGetLastError());
  k_clear_mean<<<1, 1, 0, c->st>>>(c->sc);
  MHIT_CUDA_TRY(cudaGetLastError());
  if (fieldn <= 3) {
    double* dst = fieldn == 1 ? c->U[c->cur] : (fieldn == 2 ? c->V[c->cur] : c->W[c->cur]);
    MHIT_CUDA_TRY(cudaMemcpyAsync(dst, buf.data(), fb, cudaMemcpyHostToDevice, c->st));
  } else if (fieldn == 5) {
    MHIT_CUDA_TRY(cudaMemcpyAsync(c->PHI[c->cur], buf.data(), fb, cudaMemcpyHostToDevice, c->st));
  } else {
    if (tsize(c) == 4) {
      // FP32 pressure (the incremental solve's predictor for the next step); the incremental
      // mode also keeps the file's FP64 values
      std::vector<float> pf(c->n);
      for (size_t i = 0; i < c->n; ++i) pf[i] = (float)buf[i];
      void* dst = incremental(c) ? static_cast<void*>(c->Q[c->cur]) : c->P;
      MHIT_CUDA_TRY(cudaMemcpyAsync(dst, pf.data(), c->n * 4, cudaMemcpyHostToDevice, c->st));
      if (incremental(c)) MHIT_CUDA_TRY(cudaMemcpyAsync(c->P64, buf.data(), fb, cudaMemcpyHostToDevice, c->st));
      MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
    } else {
      MHIT_CUDA_TRY(cudaMemcpyAsync(c->P, buf.data(), fb, cudaMemcpyHostToDevice, c->st));
    }
    c->p_lazy = false;
  }
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  // a field read happens at setup: the next step is an Euler step with empty history
  // (multi/main.f90:440-441; rhs_o is not part of the files); the pressure stays (a pressure
  // read is the incremental solve's predictor, whichever field is read after it)
  return reset_history(c, true);
}

// ------------------------------------------------------------------ checkpoint
// File layout (little-endian): CkptHeader, DevScalars, then the arrays in the order of
// ckpt_arrays(), each raw and complete, then the tracer table (np x 12 float64).
namespace {
struct CkptHeader {
  char magic[8];  // "MHITCKP1"
  int32_t nx, ny, nz, phiflag, partflag, poisson, np, pbytes;
  int64_t nstep;
};
constexpr char kCkptMagic[8] = {'M', 'H', 'I', 'T', 'C', 'K', 'P', '1'};

struct CkptArray {
  void* dev;
  size_t bytes;
};

std::vector<CkptArray> ckpt_arrays(mhit_ctx* c) {
  const size_t fb = c->n * sizeof(double);
  const int k = c->cur;
  std::vector<CkptArray> a = {{c->U[k], fb}, {c->V[k], fb}, {c->W[k], fb}, {c->RU, fb}, {c->RV, fb}, {c->RW, fb}};
  if (c->prm.phiflag) {
    a.push_back({c->PHI[k], fb});
    a.push_back({c->RPHI, fb});
  }
  // the pressure in the Poisson precision (incremental: the predictor the next step reads)
  a.push_back({incremental(c) ? static_cast<void*>(c->Q[k]) : c->P, c->n * tsize(c)});
  if (c->P2) a.push_back({c->P2, c->n * sizeof(float)});  // refinement: the correction
  if (incremental(c)) a.push_back({c->P64, c->n * sizeof(double)});  // incremental: the FP64 pressure
  return a;
}

struct FileCloser {
  FILE* f;
  ~FileCloser() {
    if (f) fclose(f);
  }
};
}  // namespace

int mhit_write_checkpoint(mhit_ctx* c, const char* path) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!path) return set_error(MHIT_ERR_ARG, "null path");
  if ((rc = materialise_pressure(c))) return rc;
  if ((rc = fetch_scalars(c))) return rc;
  FileCloser fc{fopen(path, "wb")};
  if (!fc.f) return set_error(MHIT_ERR_IO, std::string("cannot create ") + path);
  CkptHeader h;
  memcpy(h.magic, kCkptMagic, 8);
  h.nx = c->prm.nx;
  h.ny = c->prm.ny;
  h.nz = c->prm.nz;
  h.phiflag = c->prm.phiflag;
  h.partflag = c->prm.partflag;
  h.poisson = c->prm.poisson;
  h.np = c->np;
  h.pbytes = (int32_t)tsize(c);
  h.nstep = c->nstep;
  bool ok = fwrite(&h, sizeof(h), 1, fc.f) == 1 && fwrite(c->sc_host, sizeof(DevScalars), 1, fc.f) == 1;
  std::vector<unsigned char> buf;
  for (const CkptArray& a : ckpt_arrays(c)) {
    buf.resize(a.bytes);
    MHIT_CUDA_TRY(cudaMemcpy(buf.data(), a.dev, a.bytes, cudaMemcpyDeviceToHost));
    ok = ok && fwrite(buf.data(), 1, a.bytes, fc.f) == a.bytes;
  }
  if (c->np > 0) {
    const size_t pb = (size_t)c->np * 12 * sizeof(double);
    buf.resize(pb);
    MHIT_CUDA_TRY(cudaMemcpy(buf.data(), c->part, pb, cudaMemcpyDeviceToHost));
    ok = ok && fwrite(buf.data(), 1, pb, fc.f) == pb;
  }
  const int cl = fclose(fc.f);
  fc.f = nullptr;
  if (!ok || cl != 0) return set_error(MHIT_ERR_IO, std::string("short write to ") + path);
  return MHIT_OK;
}

int mhit_read_checkpoint(mhit_ctx* c, const char* path) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!path) return set_error(MHIT_ERR_ARG, "null path");
  FileCloser fc{fopen(path, "rb")};
  if (!fc.f) return set_error(MHIT_ERR_IO, std::string("cannot open ") + path);
  CkptHeader h;
  if (fread(&h, sizeof(h), 1, fc.f) != 1 || memcmp(h.magic, kCkptMagic, 8) != 0)
    return set_error(MHIT_ERR_IO, std::string("not a checkpoint file: ") + path);
  if (h.nx != c->prm.nx || h.ny != c->prm.ny || h.nz != c->prm.nz || h.phiflag != c->prm.phiflag ||
      h.partflag != c->prm.partflag || h.poisson != c->prm.poisson || h.pbytes != (int32_t)tsize(c) ||
      h.np < 0 || h.nstep < 0)
    return set_error(MHIT_ERR_ARG, "checkpoint was written by a context of another size or mode");
  // the whole file must be there before any device state changes: a truncated checkpoint
  // leaves the context as it was
  {
    size_t want = sizeof(CkptHeader) + sizeof(DevScalars);
    for (const CkptArray& a : ckpt_arrays(c)) want += a.bytes;
    if (c->prm.partflag) want += (size_t)h.np * 12 * sizeof(double);
    const long here = ftell(fc.f);
    if (here < 0 || fseek(fc.f, 0, SEEK_END) != 0) return set_error(MHIT_ERR_IO, std::string("cannot seek in ") + path);
    const long size = ftell(fc.f);
    if (size < 0 || fseek(fc.f, here, SEEK_SET) != 0)
      return set_error(MHIT_ERR_IO, std::string("cannot seek in ") + path);
    if ((size_t)size != want) {
      char b[160];
      snprintf(b, sizeof(b), "checkpoint holds %ld bytes, its header needs %zu: ", size, want);
      return set_error(MHIT_ERR_IO, std::string(b) + path);
    }
  }
  DevScalars s;
  if (fread(&s, sizeof(s), 1, fc.f) != 1) return set_error(MHIT_ERR_IO, std::string("short read from ") + path);
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  c->cur = 0;
  std::vector<unsigned char> buf;
  for (const CkptArray& a : ckpt_arrays(c)) {
    buf.resize(a.bytes);
    if (fread(buf.data(), 1, a.bytes, fc.f) != a.bytes)
      return set_error(MHIT_ERR_IO, std::string("short read from ") + path);
    MHIT_CUDA_TRY(cudaMemcpy(a.dev, buf.data(), a.bytes, cudaMemcpyHostToDevice));
  }
  if (c->prm.partflag) {
    const size_t pb = (size_t)h.np * 12 * sizeof(double);
    buf.resize(pb);
    if (fread(buf.data(), 1, pb, fc.f) != pb) return set_error(MHIT_ERR_IO, std::string("short read from ") + path);
    rc = mhit_upload_particles(c, h.np ? reinterpret_cast<const double*>(buf.data()) : nullptr, h.np);
    if (rc) return rc;
  }
  *c->sc_host = s;
  MHIT_CUDA_TRY(cudaMemcpy(c->sc, c->sc_host, sizeof(DevScalars), cudaMemcpyHostToDevice));
  c->nstep = h.nstep;
  c->p_lazy = false;
  return MHIT_OK;
}

// ------------------------------------------------------------------ droplet labelling
namespace {
// device buffer that only grows (kept by the context across calls)
int grow_buffer(void** p, size_t* have, size_t need) {
  if (*have >= need) return MHIT_OK;
  cudaFree(*p);
  *p = nullptr;
  *have = 0;
  MHIT_CUDA_TRY(cudaMalloc(p, need));
  *have = need;
  return MHIT_OK;
}

struct DevBuf {  // temporary device allocation freed on every return path
  void* p = nullptr;
  ~DevBuf() {
    if (p) cudaFree(p);
  }
};
}  // namespace

int mhit_label_drops(mhit_ctx* c, double thresh, int connectivity, mhit_drop* drops, int maxdrops, int* ndrops,
                     int* labels) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!c->prm.phiflag) return set_error(MHIT_ERR_STATE, "context was created with phiflag=0");
  if (connectivity != 6 && connectivity != 26) return set_error(MHIT_ERR_ARG, "connectivity must be 6 or 26");
  if (!ndrops || maxdrops < 0 || (maxdrops > 0 && !drops)) return set_error(MHIT_ERR_ARG, "bad drop buffer");
  const int nx = c->prm.nx, ny = c->prm.ny, nz = c->prm.nz;
  const int n = (int)c->n;
  const int nch = label_chunks(n);
  if ((rc = materialise_pressure(c))) return rc;  // the spectrum becomes scratch
  // scratch: the spectrum buffer (at least 4 bytes per cell, unused between steps) holds the
  // parents; the chunk counts, the error flag and the trig tables share one allocation
  const size_t trig_n = 2 * (size_t)(nx + ny + nz);
  DevBuf outb;
  const size_t small_bytes = sizeof(double) * trig_n + sizeof(int) * (nch + 1);
  if ((rc = grow_buffer(&c->lab_small, &c->lab_small_bytes, small_bytes))) return rc;
  double* trig = static_cast<double*>(c->lab_small);
  int* counts = reinterpret_cast<int*>(trig + trig_n);
  int* err = counts + nch;
  // cell centres x_i = dx/2 + (i-1) dx accumulated as post/unionfind_periodic/main.f90:294-298,
  // sin/cos(2 pi x_i / L) with L the axis period (2 pi for the cubic box)
  const double pi = 4.0 * atan(1.0), dx = 2.0 * pi / nx;
  std::vector<double> th(trig_n);
  {
    size_t o = 0;
    for (int axis = 0; axis < 3; ++axis) {
      const int na = axis == 0 ? nx : (axis == 1 ? ny : nz);
      const double L = na * dx;
      double x = dx / 2.0;
      for (int i = 0; i < na; ++i) {
        if (i > 0) x = x + dx;
        th[o + i] = sin(2.0 * pi * x / L);
        th[o + na + i] = cos(2.0 * pi * x / L);
      }
      o += 2 * (size_t)na;
    }
  }
  MHIT_CUDA_TRY(cudaMemcpyAsync(trig, th.data(), sizeof(double) * trig_n, cudaMemcpyHostToDevice, c->st));
  MHIT_CUDA_TRY(cudaMemsetAsync(err, 0, sizeof(int), c->st));
  LabelArgs a;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.phi = c->PHI[c->cur];
  a.thresh = thresh;
  a.connectivity = connectivity;
  a.lab = static_cast<int*>(c->spec);
  a.counts = counts;
  a.err = err;
  a.u = c->U[c->cur];
  a.v = c->V[c->cur];
  a.w = c->W[c->cur];
  a.sc = c->sc;
  a.trig = trig;
  a.acc = nullptr;
  a.cells = nullptr;
  a.out = nullptr;
  a.bound = c->label_bound;
  MHIT_CUDA_TRY(launch_label_components(a, c->st));
  std::vector<int> cnt(nch + 1);
  MHIT_CUDA_TRY(cudaMemcpyAsync(cnt.data(), counts, sizeof(int) * (nch + 1), cudaMemcpyDeviceToHost, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  if (cnt[nch]) return set_error(MHIT_ERR_STATE, "droplet labelling: union-find bound exceeded");
  int total = 0;
  for (int b = 0; b < nch; ++b) {  // exclusive prefix sum: first drop number of each chunk
    const int k = cnt[b];
    cnt[b] = total;
    total += k;
  }
  MHIT_CUDA_TRY(cudaMemcpyAsync(counts, cnt.data(), sizeof(int) * nch, cudaMemcpyHostToDevice, c->st));
  MHIT_CUDA_TRY(launch_label_number(a, c->st));
  const size_t nd = (size_t)std::max(total, 1);
  const size_t acc_bytes = nd * (9 * sizeof(double) + sizeof(unsigned long long));
  if ((rc = grow_buffer(&c->lab_acc, &c->lab_acc_bytes, acc_bytes))) return rc;
  a.acc = static_cast<double*>(c->lab_acc);
  a.cells = reinterpret_cast<unsigned long long*>(a.acc + nd * 9);
  MHIT_CUDA_TRY(cudaMemsetAsync(c->lab_acc, 0, acc_bytes, c->st));
  if (labels) {
    MHIT_CUDA_TRY(cudaMalloc(&outb.p, sizeof(int) * c->n));
    a.out = static_cast<int*>(outb.p);
  }
  MHIT_CUDA_TRY(launch_label_stats(a, c->st));
  std::vector<double> acc(nd * 9);
  std::vector<unsigned long long> cells(nd);
  MHIT_CUDA_TRY(cudaMemcpyAsync(acc.data(), a.acc, sizeof(double) * nd * 9, cudaMemcpyDeviceToHost, c->st));
  MHIT_CUDA_TRY(cudaMemcpyAsync(cells.data(), a.cells, sizeof(unsigned long long) * nd, cudaMemcpyDeviceToHost, c->st));
  if (labels) MHIT_CUDA_TRY(cudaMemcpyAsync(labels, a.out, sizeof(int) * c->n, cudaMemcpyDeviceToHost, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  // post/unionfind_periodic/main.f90:319-336 and the volume of :436
  const double per[3] = {nx * dx, ny * dx, nz * dx};
  for (int d = 0; d < total && d < maxdrops; ++d) {
    const double* s = &acc[(size_t)d * 9];
    mhit_drop& o = drops[d];
    o.cells = (long long)cells[d];
    o.volume = (double)cells[d] * dx * dx * dx;
    double ctr[3];
    for (int q = 0; q < 3; ++q) {
      ctr[q] = per[q] * atan2(s[2 * q], s[2 * q + 1]) / (2.0 * pi);
      if (ctr[q] < 0.0) ctr[q] = ctr[q] + per[q];
    }
    o.x = ctr[0];
    o.y = ctr[1];
    o.z = ctr[2];
    o.u = s[6] / (double)cells[d];
    o.v = s[7] / (double)cells[d];
    o.w = s[8] / (double)cells[d];
  }
  *ndrops = total;
  return MHIT_OK;
}

// ------------------------------------------------------------------ test hooks
// ------------------------------------------------------------------ initial conditions on the device
namespace {
int to_device(DevBuf& b, const std::vector<double>& v, cudaStream_t st) {
  MHIT_CUDA_TRY(cudaMalloc(&b.p, v.size() * sizeof(double)));
  MHIT_CUDA_TRY(cudaMemcpyAsync(b.p, v.data(), v.size() * sizeof(double), cudaMemcpyHostToDevice, st));
  return MHIT_OK;
}
}  // namespace

int mhit_init_taylor_green(mhit_ctx* c) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  const int nx = c->prm.nx, ny = c->prm.ny, nz = c->prm.nz, s = c->prm.yz_shift;
  const double dx = c->g.dx;
  // multi/main.f90:324-337 on the accumulated coordinates x(i) = x(i-1) + dx (:210-214), y and z
  // read s entries on (the halo-shifted labelling)
  const std::vector<double> xa = grid_coords(std::max(nx, std::max(ny, nz)) + 1, dx);
  std::vector<double> tab;
  tab.reserve(2 * (size_t)nx + 2 * (size_t)ny + nz);
  for (int i = 0; i < nx; ++i) tab.push_back(std::sin(xa[i] - dx / 2));
  for (int i = 0; i < nx; ++i) tab.push_back(std::cos(xa[i]));
  for (int j = 0; j < ny; ++j) tab.push_back(std::sin(xa[j + s] - dx / 2));
  for (int j = 0; j < ny; ++j) tab.push_back(std::cos(xa[j + s]));
  for (int k = 0; k < nz; ++k) tab.push_back(std::cos(xa[k + s]));
  DevBuf dt;
  if ((rc = to_device(dt, tab, c->st))) return rc;
  // into the current ping-pong slot: phi (when present) stays where it is
  const int k = c->cur;
  MHIT_CUDA_TRY(launch_init_tg(c->U[k], c->V[k], c->W[k], static_cast<const double*>(dt.p), nx, ny, nz, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return reset_history(c);
}

int mhit_init_velocity_modes(mhit_ctx* c, int kmax, const double* modes, double rms) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (kmax < 1 || kmax > 16 || !modes) return set_error(MHIT_ERR_ARG, "kmax must be 1..16 and modes non-null");
  if (!(rms > 0.0)) return set_error(MHIT_ERR_ARG, "rms must be positive");
  const int nx = c->prm.nx, ny = c->prm.ny, nz = c->prm.nz, s = c->prm.yz_shift;
  const int K = 2 * kmax + 1;
  const size_t k3 = (size_t)K * K * K;
  const double lx = 8.0 * std::atan(1.0);
  // scratch: the three components' modes, the exp(i k x) tables, A, B and the partial sums
  std::vector<double> cm(modes, modes + 2 * 3 * k3);
  DevBuf dcm, dA, dB, dpart;
  if ((rc = to_device(dcm, cm, c->st))) return rc;
  MHIT_CUDA_TRY(cudaMalloc(&dA.p, (size_t)K * K * nx * sizeof(Cx<double>)));
  MHIT_CUDA_TRY(cudaMalloc(&dB.p, (size_t)K * ny * nx * sizeof(Cx<double>)));
  const int npart = modes_partials(nx, ny);
  MHIT_CUDA_TRY(cudaMalloc(&dpart.p, (size_t)npart * sizeof(double)));
  std::vector<double> part(npart);
  // into the current ping-pong slot: phi (when present) stays where it is; on an error return
  // the velocity is undefined
  double* dst[3] = {c->U[c->cur], c->V[c->cur], c->W[c->cur]};
  for (int comp = 0; comp < 3; ++comp) {
    // index phases theta = (i + shift) 2 pi/n per axis (x: shift 0, y and z: yz_shift), the
    // component's own axis half a cell back (its face position, multi/main.f90:331); for a box of
    // nx dx by ny dx by nz dx the index wavenumber m_y is the physical m_y nx/ny
    auto table = [&](int n, int shift, bool face) {
      const double h = lx / n;
      std::vector<double> t(2 * (size_t)n * K);
      for (int i = 0; i < n; ++i) {
        double x = (double)(i + shift) * h;
        if (face) x = x - h / 2;
        for (int q = 0; q < K; ++q) {
          const double a = x * (double)(q - kmax);
          t[2 * ((size_t)i * K + q)] = std::cos(a);
          t[2 * ((size_t)i * K + q) + 1] = std::sin(a);
        }
      }
      return t;
    };
    DevBuf dex, dey, dez;
    if ((rc = to_device(dex, table(nx, 0, comp == 0), c->st))) return rc;
    if ((rc = to_device(dey, table(ny, s, comp == 1), c->st))) return rc;
    if ((rc = to_device(dez, table(nz, s, comp == 2), c->st))) return rc;
    ModeArgs a;
    a.nx = nx;
    a.ny = ny;
    a.nz = nz;
    a.K = K;
    a.cm = static_cast<const Cx<double>*>(dcm.p) + (size_t)comp * k3;
    a.ex = static_cast<const Cx<double>*>(dex.p);
    a.ey = static_cast<const Cx<double>*>(dey.p);
    a.ez = static_cast<const Cx<double>*>(dez.p);
    a.A = static_cast<Cx<double>*>(dA.p);
    a.Bt = static_cast<Cx<double>*>(dB.p);
    a.f = dst[comp];
    a.partials = static_cast<double*>(dpart.p);
    MHIT_CUDA_TRY(launch_init_modes(a, c->st));
    MHIT_CUDA_TRY(cudaMemcpyAsync(part.data(), dpart.p, part.size() * sizeof(double), cudaMemcpyDeviceToHost, c->st));
    MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));  // the tables are freed at the end of this iteration
    double ss = 0.0;
    for (double v : part) ss += v;
    const double mean2 = ss / (double)c->n;
    if (!(mean2 > 0.0)) return set_error(MHIT_ERR_ARG, "the modes give a zero field");
    MHIT_CUDA_TRY(launch_scale(dst[comp], c->n, rms / std::sqrt(mean2), c->st));
  }
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return reset_history(c);
}

int mhit_init_drops(mhit_ctx* c, int ndrops, const double* centres, double radius) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!c->prm.phiflag) return set_error(MHIT_ERR_STATE, "context was created with phiflag=0");
  if (ndrops < 1 || !centres || !(radius > 0.0)) return set_error(MHIT_ERR_ARG, "need ndrops >= 1, centres, radius > 0");
  const int nx = c->prm.nx, ny = c->prm.ny, nz = c->prm.nz;
  const double lx = 8.0 * std::atan(1.0);
  std::vector<double> cen(centres, centres + 3 * (size_t)ndrops);
  DevBuf dc;
  if ((rc = to_device(dc, cen, c->st))) return rc;
  // the velocity keeps its values: make its lazily removed mean explicit first
  k_apply_mean<<<148 * 4, 256, 0, c->st>>>(c->U[c->cur], c->V[c->cur], c->W[c->cur], c->n, c->sc);
  MHIT_CUDA_TRY(cudaGetLastError());
  k_clear_mean<<<1, 1, 0, c->st>>>(c->sc);
  MHIT_CUDA_TRY(cudaGetLastError());
  DropInitArgs a;
  a.phi = c->PHI[c->cur];
  a.centres = static_cast<const double*>(dc.p);
  a.nd = ndrops;
  a.nx = nx;
  a.ny = ny;
  a.nz = nz;
  a.s = c->prm.yz_shift;
  a.dx = c->g.dx;
  a.lx = lx;  // the box is 2 pi along x and n dx along y and z
  a.ly = ny == nx ? lx : a.dx * ny;
  a.lz = nz == nx ? lx : a.dx * nz;
  a.radius = radius;
  a.eps = c->g.eps;  // epsr dx
  MHIT_CUDA_TRY(launch_init_drops(a, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return reset_history(c);
}

// ------------------------------------------------------------------ energy spectrum
int mhit_energy_spectrum(mhit_ctx* c, double* E, int nbins) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!E || nbins < 1 || nbins > 4096) return set_error(MHIT_ERR_ARG, "nbins must be 1..4096 and E non-null");
  const Geo& g = c->g;
  void* spec;
  const void *tx, *ty, *tz;
  if (c->prm.poisson == MHIT_POISSON_FP64) {  // the Poisson spectrum is scratch between steps
    if ((rc = materialise_pressure(c))) return rc;
    spec = c->spec;
    tx = c->twx;
    ty = c->twy;
    tz = c->twz;
  } else {
    if ((rc = grow_buffer(&c->spec64, &c->spec64_bytes, (size_t)g.pitch * g.ny * g.nz * sizeof(Cx<double>))))
      return rc;
    if (!c->tw64[0]) {
      const int ns[3] = {g.nx, g.ny, g.nz};
      for (int q = 0; q < 3; ++q)
        if ((rc = upload_vec(&c->tw64[q], twiddles<double>(ns[q])))) return rc;
    }
    spec = c->spec64;
    tx = c->tw64[0];
    ty = c->tw64[1];
    tz = c->tw64[2];
  }
  DevBuf dpart, dE;
  MHIT_CUDA_TRY(cudaMalloc(&dpart.p, (size_t)spectrum_blocks(g) * nbins * sizeof(double)));
  MHIT_CUDA_TRY(cudaMalloc(&dE.p, (size_t)nbins * sizeof(double)));
  MHIT_CUDA_TRY(cudaMemsetAsync(dE.p, 0, (size_t)nbins * sizeof(double), c->st));
  const double* fields[3] = {c->U[c->cur], c->V[c->cur], c->W[c->cur]};
  for (int comp = 0; comp < 3; ++comp) {
    PoissonArgs a;
    a.g = g;
    a.fp32 = false;
    a.u = fields[comp];
    a.v = a.w = nullptr;
    a.real64 = true;
    a.spec = spec;
    a.p = nullptr;
    a.twx = tx;
    a.twy = ty;
    a.twz = tz;
    a.k2x = a.k2y = a.k2z = nullptr;
    a.cdiv = 0.0;
    a.ntot = (double)c->n;
    MHIT_CUDA_TRY(poisson_stage(a, PSTAGE_XFWD, c->st));
    MHIT_CUDA_TRY(poisson_stage(a, PSTAGE_YFWD, c->st));
    MHIT_CUDA_TRY(poisson_stage(a, PSTAGE_ZFWD, c->st));
    MHIT_CUDA_TRY(launch_spectrum_bin(static_cast<const Cx<double>*>(spec), g, c->sc, comp, nbins,
                                      static_cast<double*>(dpart.p), static_cast<double*>(dE.p), c->st));
  }
  MHIT_CUDA_TRY(cudaMemcpyAsync(E, dE.p, (size_t)nbins * sizeof(double), cudaMemcpyDeviceToHost, c->st));
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return MHIT_OK;
}

int mhit_debug_run_stage(mhit_ctx* c, int stage) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (stage < 0 || stage >= ST_COUNT) return set_error(MHIT_ERR_ARG, "stage out of range");
  if ((rc = materialise_pressure(c))) return rc;
  const bool first = c->nstep == 0;
  // the staged step runs every stage on its own (the x-inverse writes the pressure)
  if ((rc = enqueue_stage(c, stage, first ? 1.0 : 1.5, first ? 0.0 : 0.5, c->cur, false))) return rc;
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  return MHIT_OK;
}

int mhit_debug_set_label_bound(mhit_ctx* c, long long bound) {
  if (!c) return set_error(MHIT_ERR_ARG, "null context");
  if (bound < 0) return set_error(MHIT_ERR_ARG, "bound must be >= 0");
  c->label_bound = bound;
  return MHIT_OK;
}

int mhit_debug_set_mom_tma(mhit_ctx* c, int on) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (on != 0 && on != 1) return set_error(MHIT_ERR_ARG, "on must be 0 or 1");
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  c->mom_tma = on;
  for (int i = 0; i < 2; ++i)  // the kernel arguments are baked into the captured graphs
    if (c->gexec[i]) {
      cudaGraphExecDestroy(c->gexec[i]);
      c->gexec[i] = nullptr;
    }
  c->graph_built = false;
  return MHIT_OK;
}

int mhit_debug_commit_step(mhit_ctx* c) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  c->cur ^= 1;
  c->nstep++;
  c->p_lazy = false;
  return MHIT_OK;
}

int mhit_debug_set_fused_projection(mhit_ctx* c, int on) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (on < -1 || on > 1) return set_error(MHIT_ERR_ARG, "on must be -1, 0 or 1");
  MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  c->fuse_xc = on;
  c->gen++;  // the stage sequence is baked into captured graphs (also the ensemble's)
  for (int i = 0; i < 2; ++i)
    if (c->gexec[i]) {
      cudaGraphExecDestroy(c->gexec[i]);
      c->gexec[i] = nullptr;
    }
  c->graph_built = false;
  return MHIT_OK;
}

long long mhit_debug_buffer_len(mhit_ctx* c, int which) {
  if (!c) return -1;
  if (which == MHIT_BUF_SPEC) return (long long)c->g.pitch * c->g.ny * c->g.nz * 2;
  if (which >= 0 && which < MHIT_BUF_SPEC) return (long long)c->n;
  return -1;
}

int mhit_debug_get_buffer(mhit_ctx* c, int which, double* out) {
  int rc;
  if ((rc = check_ctx(c))) return rc;
  if (!out) return set_error(MHIT_ERR_ARG, "null buffer");
  const int cur = c->cur, nxt = cur ^ 1;
  const void* src = nullptr;
  bool typed = false;  // buffer in the Poisson precision
  size_t len = c->n;
  if (which == MHIT_BUF_P && (rc = materialise_pressure(c))) return rc;
  switch (which) {
    case MHIT_BUF_U: src = c->U[cur]; break;
    case MHIT_BUF_V: src = c->V[cur]; break;
    case MHIT_BUF_W: src = c->W[cur]; break;
    case MHIT_BUF_UN: src = c->U[nxt]; break;
    case MHIT_BUF_VN: src = c->V[nxt]; break;
    case MHIT_BUF_WN: src = c->W[nxt]; break;
    case MHIT_BUF_P:  // incremental: the FP64 pressure of the last projection
      if (incremental(c)) src = c->P64;
      else {
        src = c->P;
        typed = true;
      }
      break;
    case MHIT_BUF_PHI: src = c->PHI[cur]; break;
    case MHIT_BUF_PHIN: src = c->PHI[nxt]; break;
    case MHIT_BUF_RU: src = c->RU; break;
    case MHIT_BUF_RV: src = c->RV; break;
    case MHIT_BUF_RW: src = c->RW; break;
    case MHIT_BUF_RPHI: src = c->RPHI; break;
    case MHIT_BUF_SPEC: src = c->spec; typed = true; len = (size_t)c->g.pitch * c->g.ny * c->g.nz * 2; break;
    default: return set_error(MHIT_ERR_ARG, "unknown buffer");
  }
  if (!src) return set_error(MHIT_ERR_STATE, "buffer not allocated on this context");
  if (typed && tsize(c) == 4) {
    std::vector<float> f(len);
    MHIT_CUDA_TRY(cudaMemcpyAsync(f.data(), src, len * 4, cudaMemcpyDeviceToHost, c->st));
    MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
    for (size_t i = 0; i < len; ++i) out[i] = f[i];
  } else {
    MHIT_CUDA_TRY(cudaMemcpyAsync(out, src, len * 8, cudaMemcpyDeviceToHost, c->st));
    MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  }
  return MHIT_OK;
}

// ------------------------------------------------------------------ ensemble of boxes
// Independent boxes of uneven sizes advanced together: every step after the first is ONE
// graph launch whose graph forks the boxes' step sequences onto `nlanes` streams (boxes on
// different lanes run concurrently, boxes on one lane back to back) and joins them.
}  // extern "C"

struct mhit_ensemble {
  int nbox = 0;
  std::vector<mhit_ctx*> box;
  int dev = 0;
  cudaStream_t st = nullptr;
  int nlanes = 1;
  std::vector<cudaStream_t> lanes;
  cudaEvent_t fork = nullptr;
  std::vector<cudaEvent_t> join;
  cudaGraphExec_t gexec[2] = {nullptr, nullptr};
  bool built = false;
  std::vector<unsigned> gen;  // the boxes' graph generations the ensemble graphs were built from
  cudaEvent_t ev[2] = {nullptr, nullptr};
  // batched schedule: per class of equal-size boxes, the phase and momentum stages of the
  // class's boxes as one persistent launch each (device work queues of (box, tile x, tile y,
  // z chunk) items), then the Poisson passes and the projection of each box on the lanes
  bool batched = false;
  bool batch_ready = false;   // device argument arrays and item lists match the boxes' tuning
  int nsm = 148;
  PhaseArgs* d_pargs[2] = {nullptr, nullptr};  // per parity of the ping-pong buffers
  MomArgs* d_margs[2] = {nullptr, nullptr};
  int4* d_pitems = nullptr;   // the classes' phase items, one class after the other
  int4* d_mitems = nullptr;   // the same for the momentum stage
  int* d_counters = nullptr;  // two queue counters per class
  struct Class {
    int p0, np, m0, nm;       // offset and count of the class's phase and momentum items
  };
  std::vector<Class> cls;     // largest boxes first
  std::vector<int> box_cls;   // class of each box
  std::vector<cudaEvent_t> cls_done;  // the class's momentum launch has finished
};

// The batched schedule needs one phase variant (all boxes with the phase field share the psi
// clamp) and one momentum variant (all boxes with or all without the phase field).
static bool ens_batchable(const mhit_ensemble* e) {
  for (const mhit_ctx* c : e->box)
    if (c->prm.phiflag != e->box[0]->prm.phiflag || c->prm.acdi_clamp != e->box[0]->prm.acdi_clamp) return false;
  return true;
}

static void ens_free_batch(mhit_ensemble* e) {
  if (e->st) cudaStreamSynchronize(e->st);  // no step in flight may still read the arrays
  for (int i = 0; i < 2; ++i) {
    cudaFree(e->d_pargs[i]);
    cudaFree(e->d_margs[i]);
    e->d_pargs[i] = nullptr;
    e->d_margs[i] = nullptr;
  }
  cudaFree(e->d_pitems);
  cudaFree(e->d_mitems);
  cudaFree(e->d_counters);
  e->d_pitems = e->d_mitems = nullptr;
  e->d_counters = nullptr;
  for (cudaEvent_t v : e->cls_done) cudaEventDestroy(v);
  e->cls_done.clear();
  e->cls.clear();
  e->box_cls.clear();
  e->batch_ready = false;
}

// Device copies of every box's phase and momentum arguments (both parities; the step's alpha,
// beta come with the launch) and the work items of each class of equal-size boxes, the classes
// largest boxes first.
static int ens_prepare_batch(mhit_ensemble* e) {
  if (e->batch_ready) return MHIT_OK;
  ens_free_batch(e);
  std::vector<size_t> sizes;
  for (const mhit_ctx* c : e->box)
    if (std::find(sizes.begin(), sizes.end(), c->n) == sizes.end()) sizes.push_back(c->n);
  std::sort(sizes.begin(), sizes.end(), std::greater<size_t>());
  e->box_cls.assign(e->nbox, 0);
  for (int b = 0; b < e->nbox; ++b)
    e->box_cls[b] = (int)(std::find(sizes.begin(), sizes.end(), e->box[b]->n) - sizes.begin());
  std::vector<int4> pit, mit;
  std::vector<PhaseArgs> pa[2];
  std::vector<MomArgs> ma[2];
  for (int b = 0; b < e->nbox; ++b) {
    mhit_ctx* c = e->box[b];
    for (int par = 0; par < 2; ++par) {
      PhaseArgs p = phase_args(c, 1.0, 0.0, par);
      p.zchunk = phase_zchunk(c->g, c->zchunk_phase);
      pa[par].push_back(p);
      MomArgs m = mom_args(c, 1.0, 0.0, par);
      m.zchunk = mom_zchunk(c->g, c->zchunk_mom);
      m.tma = 0;  // the tensor maps would be read from device memory: per-thread ring copies
      ma[par].push_back(m);
    }
  }
  for (size_t k = 0; k < sizes.size(); ++k) {
    mhit_ensemble::Class cl{(int)pit.size(), 0, (int)mit.size(), 0};
    for (int b = 0; b < e->nbox; ++b) {
      if (e->box_cls[b] != (int)k) continue;
      const mhit_ctx* c = e->box[b];
      if (c->prm.phiflag) {
        const dim3 gp = phase_grid(c->g, pa[0][b].zchunk);
        for (unsigned z = 0; z < gp.z; ++z)
          for (unsigned y = 0; y < gp.y; ++y)
            for (unsigned x = 0; x < gp.x; ++x) pit.push_back(make_int4(b, (int)x, (int)y, (int)z));
      }
      const dim3 gm = mom_grid(c->g, ma[0][b].zchunk);
      for (unsigned z = 0; z < gm.z; ++z)
        for (unsigned y = 0; y < gm.y; ++y)
          for (unsigned x = 0; x < gm.x; ++x) mit.push_back(make_int4(b, (int)x, (int)y, (int)z));
    }
    cl.np = (int)pit.size() - cl.p0;
    cl.nm = (int)mit.size() - cl.m0;
    e->cls.push_back(cl);
    cudaEvent_t ev;
    MHIT_CUDA_TRY(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    e->cls_done.push_back(ev);
  }
  int rc;
  for (int par = 0; par < 2; ++par) {
    if ((rc = upload_vec((void**)&e->d_pargs[par], pa[par]))) return rc;
    if ((rc = upload_vec((void**)&e->d_margs[par], ma[par]))) return rc;
  }
  if (!pit.empty() && (rc = upload_vec((void**)&e->d_pitems, pit))) return rc;
  if ((rc = upload_vec((void**)&e->d_mitems, mit))) return rc;
  MHIT_CUDA_TRY(cudaMalloc(&e->d_counters, 2 * e->cls.size() * sizeof(int)));
  e->batch_ready = true;
  return MHIT_OK;
}

static void ens_drop_graphs(mhit_ensemble* e) {
  for (int i = 0; i < 2; ++i)
    if (e->gexec[i]) {
      cudaGraphExecDestroy(e->gexec[i]);
      e->gexec[i] = nullptr;
    }
  e->built = false;
  e->batch_ready = false;  // z chunks or buffers may have changed
}

static int ens_set_lanes(mhit_ensemble* e, int nlanes) {
  if (nlanes < 1) nlanes = 1;
  if (nlanes > e->nbox) nlanes = e->nbox;
  MHIT_CUDA_TRY(cudaStreamSynchronize(e->st));
  for (cudaStream_t s : e->lanes) cudaStreamDestroy(s);
  for (cudaEvent_t v : e->join) cudaEventDestroy(v);
  e->lanes.assign(nlanes, nullptr);
  e->join.assign(nlanes, nullptr);
  for (int l = 0; l < nlanes; ++l) {
    MHIT_CUDA_TRY(cudaStreamCreateWithFlags(&e->lanes[l], cudaStreamNonBlocking));
    MHIT_CUDA_TRY(cudaEventCreateWithFlags(&e->join[l], cudaEventDisableTiming));
  }
  e->nlanes = nlanes;
  ens_drop_graphs(e);
  return MHIT_OK;
}

// One ensemble step on e->st (captured or eager): fork, per-box sequences on lanes, join.  In the
// batched schedule the tracers of all boxes run first on e->st; then each class of equal-size
// boxes runs its phase and momentum stages as one persistent launch each on a lane of its own
// (the last lanes), and each box's Poisson passes and projection follow on its lane as soon as
// its class's momentum launch is done, so small boxes start their Poisson solves while large
// boxes are still in their stencils.
static int ens_enqueue(mhit_ensemble* e, double alpha, double beta, int cur) {
  int first = 0;
  if (e->batched) {
    int rc;
    // the device argument arrays are built before any capture (they allocate)
    if (!e->batch_ready) return set_error(MHIT_ERR_STATE, "batched ensemble arguments not prepared");
    for (mhit_ctx* c : e->box) {
      cudaStream_t saved = c->st;
      c->st = e->st;
      rc = enqueue_stage(c, ST_TRACER, alpha, beta, cur, fused_xc(c));
      c->st = saved;
      if (rc) return rc;
    }
    first = ST_XFWD;
  }
  MHIT_CUDA_TRY(cudaEventRecord(e->fork, e->st));
  for (int l = 0; l < e->nlanes; ++l) MHIT_CUDA_TRY(cudaStreamWaitEvent(e->lanes[l], e->fork, 0));
  if (e->batched) {
    for (size_t k = 0; k < e->cls.size(); ++k) {
      const mhit_ensemble::Class& cl = e->cls[k];
      cudaStream_t lane = e->lanes[e->nlanes - 1 - (int)(k % e->nlanes)];
      if (cl.np) {
        BatchArgs<PhaseArgs> pb{e->d_pargs[cur], e->d_pitems + cl.p0, cl.np, e->d_counters + 2 * k, alpha, beta};
        MHIT_CUDA_TRY(launch_phase_batch(pb, e->box[0]->prm.acdi_clamp != 0, e->nsm, lane));
      }
      BatchArgs<MomArgs> mb{e->d_margs[cur], e->d_mitems + cl.m0, cl.nm, e->d_counters + 2 * k + 1, alpha, beta};
      MHIT_CUDA_TRY(launch_mom_batch(mb, e->box[0]->prm.phiflag != 0, e->nsm, lane));
      MHIT_CUDA_TRY(cudaEventRecord(e->cls_done[k], lane));
    }
  }
  for (int b = 0; b < e->nbox; ++b) {
    mhit_ctx* c = e->box[b];
    cudaStream_t saved = c->st;
    c->st = e->lanes[b % e->nlanes];
    if (e->batched) MHIT_CUDA_TRY(cudaStreamWaitEvent(c->st, e->cls_done[e->box_cls[b]], 0));
    int rc = MHIT_OK;
    for (int s = first; s < ST_COUNT && rc == MHIT_OK; ++s) rc = enqueue_stage(c, s, alpha, beta, cur, fused_xc(c));
    c->st = saved;
    if (rc) return rc;
  }
  for (int l = 0; l < e->nlanes; ++l) {
    MHIT_CUDA_TRY(cudaEventRecord(e->join[l], e->lanes[l]));
    MHIT_CUDA_TRY(cudaStreamWaitEvent(e->st, e->join[l], 0));
  }
  return MHIT_OK;
}

static int ens_build(mhit_ensemble* e) {
  int rc0;
  if (e->batched && (rc0 = ens_prepare_batch(e))) return rc0;
  for (int par = 0; par < 2; ++par) {
    cudaGraph_t graph;
    MHIT_CUDA_TRY(cudaStreamBeginCapture(e->st, cudaStreamCaptureModeThreadLocal));
    int rc = ens_enqueue(e, 1.5, 0.5, par);
    cudaError_t err = cudaStreamEndCapture(e->st, &graph);
    if (rc) return rc;
    if (err != cudaSuccess) return set_cuda_error(err, "cudaStreamEndCapture (ensemble)", __FILE__, __LINE__);
    err = cudaGraphInstantiate(&e->gexec[par], graph, 0);
    cudaGraphDestroy(graph);
    if (err != cudaSuccess) return set_cuda_error(err, "cudaGraphInstantiate (ensemble)", __FILE__, __LINE__);
  }
  e->built = true;
  e->gen.clear();
  for (mhit_ctx* c : e->box) e->gen.push_back(c->gen);
  return MHIT_OK;
}

static int ens_enqueue_steps(mhit_ensemble* e, int nsteps) {
  for (int s = 0; s < nsteps; ++s) {
    const long long n0 = e->box[0]->nstep;
    const int cur = e->box[0]->cur;
    for (mhit_ctx* c : e->box)
      if (c->nstep != n0 || c->cur != cur)
        return set_error(MHIT_ERR_STATE, "ensemble boxes are at different steps (upload or step all of them together)");
    int rc;
    if (n0 == 0) {
      if (e->batched && (rc = ens_prepare_batch(e))) return rc;
      rc = ens_enqueue(e, 1.0, 0.0, cur);  // Euler first step, multi/main.f90:440-441
    } else {
      // a box whose captured arguments changed (tracers uploaded) invalidates the ensemble graphs
      for (size_t b = 0; e->built && b < e->box.size(); ++b)
        if (e->gen.size() != e->box.size() || e->gen[b] != e->box[b]->gen) ens_drop_graphs(e);
      if (!e->built && (rc = ens_build(e))) return rc;
      MHIT_CUDA_TRY(cudaGraphLaunch(e->gexec[cur], e->st));
      rc = MHIT_OK;
    }
    if (rc) return rc;
    for (mhit_ctx* c : e->box) {
      c->cur ^= 1;
      c->nstep++;
      c->p_lazy = fused_xc(c);
    }
  }
  return MHIT_OK;
}

static int ens_check_flags(mhit_ensemble* e) {
  MHIT_CUDA_TRY(cudaStreamSynchronize(e->st));
  for (int b = 0; b < e->nbox; ++b) {
    int rc;
    if ((rc = fetch_scalars(e->box[b]))) return rc;
    const int flag = e->box[b]->sc_host->flag;
    if (flag & 1) return set_error(MHIT_ERR_NAN, "NaN in the velocity field of ensemble box " + std::to_string(b));
    if (flag & 2) return set_error(MHIT_ERR_CFL, "CFL > 7 in ensemble box " + std::to_string(b));
  }
  return MHIT_OK;
}

// zero fields, empty history, Euler next (used around the autotuner's throwaway steps)
static int reset_state(mhit_ctx* c) {
  const size_t fb = c->n * sizeof(double);
  for (int i = 0; i < 2; ++i) {
    MHIT_CUDA_TRY(cudaMemsetAsync(c->U[i], 0, fb, c->st));
    MHIT_CUDA_TRY(cudaMemsetAsync(c->V[i], 0, fb, c->st));
    MHIT_CUDA_TRY(cudaMemsetAsync(c->W[i], 0, fb, c->st));
    if (c->PHI[i]) MHIT_CUDA_TRY(cudaMemsetAsync(c->PHI[i], 0, fb, c->st));
  }
  c->cur = 0;
  return reset_history(c);
}

extern "C" {

int mhit_ensemble_create(const mhit_params* params, int nbox, mhit_ensemble** out) {
  if (!params || !out || nbox < 1) return set_error(MHIT_ERR_ARG, "need at least one box");
  *out = nullptr;
  for (int b = 1; b < nbox; ++b)
    if (params[b].device != params[0].device) return set_error(MHIT_ERR_ARG, "all ensemble boxes must use one device");
  mhit_ensemble* e = new mhit_ensemble();
  e->nbox = nbox;
  e->dev = params[0].device;
  int rc = MHIT_OK;
  for (int b = 0; b < nbox && rc == MHIT_OK; ++b) {
    mhit_ctx* c = nullptr;
    rc = mhit_init(&params[b], &c);
    if (rc == MHIT_OK) e->box.push_back(c);
  }
  if (rc == MHIT_OK) {
    cudaError_t err = cudaStreamCreateWithFlags(&e->st, cudaStreamNonBlocking);
    if (err == cudaSuccess) err = cudaEventCreateWithFlags(&e->fork, cudaEventDisableTiming);
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev[0]);
    if (err == cudaSuccess) err = cudaEventCreate(&e->ev[1]);
    if (err != cudaSuccess) rc = set_cuda_error(err, "ensemble stream/events", __FILE__, __LINE__);
  }
  if (rc == MHIT_OK) rc = ens_set_lanes(e, nbox);
  if (rc == MHIT_OK) {
    cudaDeviceGetAttribute(&e->nsm, cudaDevAttrMultiProcessorCount, e->dev);
    e->batched = ens_batchable(e);  // the autotuner may switch back to per-box lanes
  }
  if (rc) {
    std::string keep = g_err;
    mhit_ensemble_destroy(e);
    g_err = keep;
    return rc;
  }
  *out = e;
  return MHIT_OK;
}

void mhit_ensemble_destroy(mhit_ensemble* e) {
  if (!e) return;
  cudaSetDevice(e->dev);
  if (e->st) cudaStreamSynchronize(e->st);
  ens_drop_graphs(e);
  ens_free_batch(e);  // before its stream goes
  for (cudaStream_t s : e->lanes) cudaStreamDestroy(s);
  for (cudaEvent_t v : e->join) cudaEventDestroy(v);
  if (e->fork) cudaEventDestroy(e->fork);
  for (int i = 0; i < 2; ++i)
    if (e->ev[i]) cudaEventDestroy(e->ev[i]);
  if (e->st) cudaStreamDestroy(e->st);
  for (mhit_ctx* c : e->box) mhit_destroy(c);
  delete e;
}

int mhit_ensemble_box(mhit_ensemble* e, int b, mhit_ctx** ctx) {
  if (!e || !ctx || b < 0 || b >= e->nbox) return set_error(MHIT_ERR_ARG, "box index out of range");
  *ctx = e->box[b];
  return MHIT_OK;
}

int mhit_ensemble_step(mhit_ensemble* e, int nsteps) {
  if (!e || nsteps < 0) return set_error(MHIT_ERR_ARG, "bad argument");
  MHIT_CUDA_TRY(cudaSetDevice(e->dev));
  // fields uploaded through a box's own stream must be complete before the ensemble stream runs
  for (mhit_ctx* c : e->box) MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  int rc;
  if ((rc = ens_enqueue_steps(e, nsteps))) return rc;
  return ens_check_flags(e);
}

int mhit_ensemble_time_steps(mhit_ensemble* e, int nsteps, double* ms) {
  if (!e || !ms || nsteps < 0) return set_error(MHIT_ERR_ARG, "bad argument");
  MHIT_CUDA_TRY(cudaSetDevice(e->dev));
  for (mhit_ctx* c : e->box) MHIT_CUDA_TRY(cudaStreamSynchronize(c->st));
  MHIT_CUDA_TRY(cudaEventRecord(e->ev[0], e->st));
  int rc;
  if ((rc = ens_enqueue_steps(e, nsteps))) return rc;
  MHIT_CUDA_TRY(cudaEventRecord(e->ev[1], e->st));
  MHIT_CUDA_TRY(cudaEventSynchronize(e->ev[1]));
  float f = 0.f;
  MHIT_CUDA_TRY(cudaEventElapsedTime(&f, e->ev[0], e->ev[1]));
  *ms = f;
  return MHIT_OK;
}

// Autotuner: for every class of equal boxes (grid, phase field on/off) time the z-chunk of
// k_phase and k_mom over {8, 16, 32, 64} on the first box of the class (one profiled step per
// candidate, best of `trials`), then time whole ensemble steps for 1, 2, 4, 8, ... lanes and
// keep the fastest; then time the batched schedule with uniform z chunks of 32, 64 and 128
// planes on those lanes and on one lane per box, and keep it if it is faster.  The timing
// steps run on zeroed fields and are thrown away: every box is left zeroed with an empty
// history, so call this before uploading the initial fields.
int mhit_ensemble_autotune(mhit_ensemble* e, int trials, int* nlanes_out) {
  if (!e) return set_error(MHIT_ERR_ARG, "null ensemble");
  if (trials < 1) trials = 1;
  MHIT_CUDA_TRY(cudaSetDevice(e->dev));
  int rc;
  for (mhit_ctx* c : e->box)
    if ((rc = reset_state(c))) return rc;
  const int cand[4] = {8, 16, 32, 64};
  std::vector<bool> done(e->nbox, false);
  for (int b = 0; b < e->nbox; ++b) {
    if (done[b]) continue;
    mhit_ctx* c = e->box[b];
    int best_p = 0, best_m = 0;
    double tp = 1e30, tm = 1e30;
    for (int q = 0; q < 4; ++q) {
      if (cand[q] > c->g.nz) continue;
      c->zchunk_phase = c->zchunk_mom = cand[q];
      double bp = 1e30, bm = 1e30;
      for (int t = 0; t < trials + 1; ++t) {
        double ms[ST_COUNT];
        int n = ST_COUNT;
        if ((rc = mhit_profile_step(c, ms, nullptr, &n))) return rc;
        if (t == 0) continue;  // first step after a reset is Euler
        if (ms[ST_PHASE] >= 0) bp = std::min(bp, ms[ST_PHASE]);
        bm = std::min(bm, ms[ST_MOM]);
      }
      if (bp < tp) {
        tp = bp;
        best_p = cand[q];
      }
      if (bm < tm) {
        tm = bm;
        best_m = cand[q];
      }
    }
    for (int o = b; o < e->nbox; ++o) {
      mhit_ctx* d = e->box[o];
      if (d->g.nx == c->g.nx && d->g.ny == c->g.ny && d->g.nz == c->g.nz && d->prm.phiflag == c->prm.phiflag) {
        d->zchunk_phase = best_p;
        d->zchunk_mom = best_m;
        done[o] = true;
      }
    }
    if ((rc = reset_state(c))) return rc;
  }
  int best_l = e->nbox;
  double best_t = 1e30;
  for (int nl = 1;; nl *= 2) {
    const int lanes = std::min(nl, e->nbox);
    if ((rc = ens_set_lanes(e, lanes))) return rc;
    for (mhit_ctx* c : e->box)
      if ((rc = reset_state(c))) return rc;
    double ms = 0.0;
    if ((rc = ens_enqueue_steps(e, 2))) return rc;  // Euler + graph build
    if ((rc = mhit_ensemble_time_steps(e, 2 * trials, &ms))) return rc;
    if (ms < best_t) {
      best_t = ms;
      best_l = lanes;
    }
    if (lanes == e->nbox) break;
  }
  if ((rc = ens_set_lanes(e, best_l))) return rc;
  // the batched schedule (phase and momentum of all boxes as one persistent launch each) with
  // uniform z chunks and the same lanes for the Poisson passes; kept if it beats the lanes
  if (ens_batchable(e)) {
    std::vector<int> zp(e->nbox), zm(e->nbox);
    for (int b = 0; b < e->nbox; ++b) {
      zp[b] = e->box[b]->zchunk_phase;
      zm[b] = e->box[b]->zchunk_mom;
    }
    const int bcand[3] = {32, 64, 128};
    const int lcand[2] = {best_l, e->nbox};
    int best_z = 0, best_bl = best_l;
    double best_bt = 1e30;
    e->batched = true;
    for (int li = 0; li < (best_l == e->nbox ? 1 : 2); ++li) {
      if ((rc = ens_set_lanes(e, lcand[li]))) return rc;
      for (int q = 0; q < 3; ++q) {
        for (mhit_ctx* c : e->box) {
          c->zchunk_phase = c->zchunk_mom = std::min(bcand[q], c->g.nz);
          if ((rc = reset_state(c))) return rc;
        }
        ens_drop_graphs(e);
        double ms = 0.0;
        if ((rc = ens_enqueue_steps(e, 2))) return rc;
        if ((rc = mhit_ensemble_time_steps(e, 2 * trials, &ms))) return rc;
        if (ms < best_bt) {
          best_bt = ms;
          best_z = bcand[q];
          best_bl = lcand[li];
        }
      }
    }
    e->batched = best_bt < best_t;
    if ((rc = ens_set_lanes(e, e->batched ? best_bl : best_l))) return rc;
    if (nlanes_out) *nlanes_out = e->nlanes;
    for (int b = 0; b < e->nbox; ++b) {
      mhit_ctx* c = e->box[b];
      c->zchunk_phase = e->batched ? std::min(best_z, c->g.nz) : zp[b];
      c->zchunk_mom = e->batched ? std::min(best_z, c->g.nz) : zm[b];
    }
    ens_drop_graphs(e);
  } else {
    e->batched = false;
  }
  for (mhit_ctx* c : e->box)
    if ((rc = reset_state(c))) return rc;
  if (nlanes_out && !e->batched) *nlanes_out = best_l;
  return MHIT_OK;
}

int mhit_ensemble_set_batched(mhit_ensemble* e, int on) {
  if (!e || (on != 0 && on != 1)) return set_error(MHIT_ERR_ARG, "on must be 0 or 1");
  if (on && !ens_batchable(e))
    return set_error(MHIT_ERR_ARG, "the batched schedule needs equal phiflag and acdi_clamp in every box");
  MHIT_CUDA_TRY(cudaSetDevice(e->dev));
  MHIT_CUDA_TRY(cudaStreamSynchronize(e->st));
  e->batched = on != 0;
  ens_drop_graphs(e);
  return MHIT_OK;
}

int mhit_ensemble_batched(mhit_ensemble* e, int* on) {
  if (!e || !on) return set_error(MHIT_ERR_ARG, "null argument");
  *on = e->batched ? 1 : 0;
  return MHIT_OK;
}

int mhit_ensemble_tuning(mhit_ensemble* e, int* nlanes, int* zchunk_phase, int* zchunk_mom) {
  if (!e) return set_error(MHIT_ERR_ARG, "null ensemble");
  if (nlanes) *nlanes = e->nlanes;
  for (int b = 0; b < e->nbox; ++b) {
    if (zchunk_phase) zchunk_phase[b] = e->box[b]->zchunk_phase;
    if (zchunk_mom) zchunk_mom[b] = e->box[b]->zchunk_mom;
  }
  return MHIT_OK;
}

}  // extern "C"
