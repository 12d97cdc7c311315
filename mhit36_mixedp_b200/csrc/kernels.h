// Host-side launchers of the timestep kernels (internal to libmhit_b200.so).
#pragma once
#include <cuda.h>
#include <cuda_runtime.h>

#include <string>

#include "../../include/mhit_b200.h"
#include "common.cuh"

namespace mhit {

int set_error(int code, const std::string& msg);
int set_cuda_error(cudaError_t e, const char* expr, const char* file, int line);

struct ZsolveTc;  // tensor-core 512-point z solve: tensor map of the spectrum, DFT-matrix image, twiddles

// the driver's cuTensorMapEncodeTiled, reached through the runtime (the library links only cudart);
// nullptr when the driver does not provide it
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);
EncodeTiledFn tensor_map_encoder();

// ---------------------------------------------------------------- Poisson
enum { PSTAGE_XFWD = 0, PSTAGE_YFWD, PSTAGE_ZSOLVE, PSTAGE_YINV, PSTAGE_XINV, PSTAGE_COUNT };
constexpr int PSTAGE_ZFWD = PSTAGE_COUNT + 1;  // forward z transform alone (energy spectrum), not a step stage

struct PoissonArgs {
  Geo g;
  bool fp32;
  const double *u, *v, *w;  // u* (input of the divergence)
  void* spec;               // Cx<T>[nz][ny][pitch]
  void* p;                  // T[nz][ny][nx]
  const void *twx, *twy, *twz;  // exp(-2 pi i m/n) tables, one per axis, in T
  const double *k2x, *k2y, *k2z;
  double cdiv;  // rho*dxi/dt
  double ntot;  // nx*ny*nz
  // non-null: x-forward transforms the FP64 residual rho/dt div(u*) - L_h presid of this FP32
  // pressure (refinement sweep, incremental solve)
  const float* presid = nullptr;
  // non-null: x-inverse adds its transform to this FP32 predictor in FP64, writes the sum to p64
  // and its FP32 rounding to qout (incremental solve; qout null: p64 only)
  const float* qin = nullptr;
  float* qout = nullptr;
  double* p64 = nullptr;
  bool real64 = false;           // x-forward transforms the FP64 field u (energy spectrum)
  const ZsolveTc* tcz = nullptr;  // non-null (FP32, nz = 512): the z solve runs on the tensor cores
  DevScalars* sc = nullptr;       // flag word for the tensor-core z solve's bounded waits
};
bool zsolve_tc_supported(const Geo& g);
int zsolve_tc_create(const Geo& g, void* spec, ZsolveTc** out);
void zsolve_tc_destroy(ZsolveTc* z);
cudaError_t launch_zsolve_tc(const ZsolveTc* z, const PoissonArgs& a, DevScalars* sc, cudaStream_t st);

cudaError_t launch_combine(const float* p32, const float* d32, double* p64, size_t n, cudaStream_t st);
cudaError_t poisson_stage(const PoissonArgs& a, int stage, cudaStream_t st);
bool poisson_size_supported(int n, bool is_x);

// ---------------------------------------------------------------- phase field
struct PhaseArgs {
  Geo g;
  const double* phi;    // phi^n
  const double *u, *v, *w;
  double* phin;         // phi^{n+1}
  double* rphio;        // rhsphi_o (read, then overwritten)
  const DevScalars* sc;
  double alpha, beta;
  int clamp;            // 1: phi clamped to [0,1] before the log
  int zchunk;           // z planes per block (0: default)
  double dta = 0, dtb = 0;  // dt alpha, dt beta (set by launch_phase)
};
cudaError_t launch_phase(const PhaseArgs& a, cudaStream_t st);

// A stage of many boxes in one launch: persistent blocks take work items (box, tile x, tile y,
// z chunk) from a device queue (counter, reset by the launcher) and run the box's tile with
// args[box] (device memory) and the step's alpha, beta.
template <typename A> struct BatchArgs {
  const A* args;
  const int4* items;
  int nitems;
  int* counter;
  double alpha, beta;
};
int phase_zchunk(const Geo& g, int requested);  // the z chunk launch_phase uses
dim3 phase_grid(const Geo& g, int zc);           // its tiles: x, y, z chunk
cudaError_t launch_phase_batch(const BatchArgs<PhaseArgs>& b, bool clamp, int nsm, cudaStream_t st);

// ---------------------------------------------------------------- momentum
struct MomArgs {
  Geo g;
  const double *u, *v, *w;   // u^n (stored; mean subtracted on read)
  double *un, *vn, *wn;      // u*
  double *ru, *rv, *rw;      // rhs_o (read, then overwritten)
  const double* phi;         // phi^{n+1} or nullptr
  const double* tabs;        // sx,cx (nx) sy,cy (ny) sz,cz (nz)
  const DevScalars* sc;
  double alpha, beta;
  int zchunk;                // z planes per block (0: default)
  // TMA tensor maps of u, v, w and phi^{n+1} (mom_field_maps); when `tma` is set the blocks whose
  // rings need no periodic wrap in x and y fill them with TMA boxes instead of per-thread copies
  int tma = 0;
  CUtensorMap tmu, tmv, tmw, tmphi;
};
cudaError_t launch_mom(const MomArgs& a, cudaStream_t st);
int mom_zchunk(const Geo& g, int requested);  // the z chunk launch_mom uses
dim3 mom_grid(const Geo& g, int zc);           // its tiles: x, y, z chunk
cudaError_t launch_mom_batch(const BatchArgs<MomArgs>& b, bool phi, int nsm, cudaStream_t st);
// tensor map of an x-fastest nx*ny*nz float64 field with the ring box of k_mom (36 x 10 for the
// velocity, 36 x 11 for phi)
int mom_field_map(CUtensorMap* map, const double* field, int nx, int ny, int nz, bool phi);

// ---------------------------------------------------------------- projection + reductions
struct CorrectArgs {
  Geo g;
  double *u, *v, *w;  // u* in, u** out (in place)
  const void* p;      // float or double pressure
  bool fp32;
  const float* pd = nullptr;  // refinement: the FP32 correction; the pressure is p + pd
  double* partials;   // [nblocks][6]
  int nblocks;
  DevScalars* sc;
};
cudaError_t launch_correct(const CorrectArgs& a, cudaStream_t st);
int correct_blocks(const Geo& g);
// k_finalize: the projection's partial sums/maxima -> mean, gumax, cfl, flags (fixed order)
cudaError_t launch_finalize(const double* partials, int nblocks, const Geo& g, DevScalars* sc, cudaStream_t st);

// the inverse x transform fused with the projection (the pressure stays on chip): u*, v*, w*
// projected in place from the y-inverted spectrum, partial sums/maxima as k_correct, then
// k_finalize.  The FP32 modes transform in FP32; qold non-null selects the incremental solve
// (pressure = qold + delta in FP64, fl32 of it to qnew).
struct XcArgs {
  Geo g;
  bool fp32;
  const void* spec;           // Cx<T>[nz][ny][pitch] after the y inverse
  const void* twx;            // exp(-2 pi i m/nx) in T
  double *u, *v, *w;          // u* in, u** out
  const float* qold = nullptr;
  float* qnew = nullptr;
  double* partials;           // [xc_blocks(g)][6]
  DevScalars* sc;
  int zc = 0;                 // z planes per block (0: default)
};
cudaError_t launch_xinv_correct(const XcArgs& a, cudaStream_t st);
int xc_blocks(const Geo& g, int zc);

// on-demand diagnostics of the current velocity: max|div|, KE, dissipation
struct DiagArgs {
  Geo g;
  const double *u, *v, *w;
  double* partials;  // [nblocks][4]
  int nblocks;
  DevScalars* sc;
  double nu, dxd;    // viscosity and spacing used by the dissipation formula
};
cudaError_t launch_diag(const DiagArgs& a, cudaStream_t st);

// ---------------------------------------------------------------- tracers
struct TracerArgs {
  Geo g;
  double* part;  // SoA [12][npmax]: tag,x,y,z,u,v,w,phi,u1,v1,w1,phi1
  int np, npmax;
  const double *u, *v, *w;
  const DevScalars* sc;
  double alpha, beta, lx;
  int interp;     // 0: 1-D linear (reference), 1: trilinear
  int yz_shift;
};
cudaError_t launch_tracer(const TracerArgs& a, cudaStream_t st);

// ---------------------------------------------------------------- utilities
cudaError_t launch_fill(double* p, size_t n, double v, cudaStream_t st);

// ---------------------------------------------------------------- droplet labelling
struct LabelArgs {
  int nx, ny, nz;
  const double* phi;
  double thresh;
  int connectivity;             // 6 or 26
  int* lab;                     // n ints of scratch: parents, then the drop encoding
  int* counts;                  // roots per chunk of cells, then the chunks' first drop numbers
  int* err;                     // set when a bounded union-find loop ran out
  const double *u, *v, *w;      // stored velocity (lazy mean in sc)
  const DevScalars* sc;
  const double* trig;           // sin, cos of the cell centres per axis (x, y, z)
  double* acc;                  // [ndrops][9]
  unsigned long long* cells;    // [ndrops]
  int* out;                     // label field (0 background, 1.. drop) or nullptr
  long long bound = 0;          // iteration bound of the union-find loops (0: the cell count)
};
int label_chunks(int n);
cudaError_t launch_label_components(const LabelArgs& a, cudaStream_t st);  // init, merge, flatten, count
cudaError_t launch_label_number(const LabelArgs& a, cudaStream_t st);      // counts must hold offsets
cudaError_t launch_label_stats(const LabelArgs& a, cudaStream_t st);

// ---------------------------------------------------------------- initial conditions
cudaError_t launch_init_tg(double* u, double* v, double* w, const double* tab, int nx, int ny, int nz,
                           cudaStream_t st);
struct ModeArgs {
  int nx, ny, nz, K;             // K = 2 kmax + 1 wavenumbers per axis
  const Cx<double>* cm;          // mode amplitudes [kz][ky][kx] of one component
  const Cx<double>* ex;          // exp(i k x) tables [nx][K], [ny][K], [nz][K]
  const Cx<double>* ey;
  const Cx<double>* ez;
  Cx<double>* A;                 // scratch [K][K][nx]
  Cx<double>* Bt;                // scratch [K][ny][nx]
  double* f;                     // output field
  double* partials;              // modes_partials(nx, ny) sums of f^2
};
int modes_partials(int nx, int ny);
cudaError_t launch_init_modes(const ModeArgs& a, cudaStream_t st);
cudaError_t launch_scale(double* f, size_t n, double s, cudaStream_t st);
struct DropInitArgs {
  double* phi;
  const double* centres;  // [nd][3]
  int nd, nx, ny, nz, s;
  double dx, lx, ly, lz, radius, eps;
};
cudaError_t launch_init_drops(const DropInitArgs& a, cudaStream_t st);
cudaError_t launch_init_particles(double* part, int np, unsigned long long seed, double lx, double ly, double lz,
                                  cudaStream_t st);

// ---------------------------------------------------------------- energy spectrum
int spectrum_blocks(const Geo& g);
// adds the shell energies of one component's FP64 half spectrum to E[0..nbins) (device);
// partials holds spectrum_blocks(g) * nbins doubles
cudaError_t launch_spectrum_bin(const Cx<double>* spec, const Geo& g, const DevScalars* sc, int comp, int nbins,
                                double* partials, double* E, cudaStream_t st);

}  // namespace mhit
