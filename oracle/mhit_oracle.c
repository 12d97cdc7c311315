/*
 * C/OpenMP restatement of the MHIT36 timestep loop (TEST INFRASTRUCTURE ONLY).
 *
 * The CPU baseline and the large-size checker: the same algorithm as oracle/mhit_oracle.py,
 * i.e. one rank of multi/main.f90:456-1007 (aroccon/MHIT36_mixedp) with periodic indexing in
 * place of halo planes, structured pass by pass as the reference (psidi/tanh_psi/normals/
 * fxst arrays materialised, one loop nest per OpenACC region).  Built with
 * -ffp-contract=off so the elementwise arithmetic rounds exactly as the Fortran expressions
 * (and as NumPy).  The cuFFT plans (multi/main.f90:187-205) are replaced by an own Stockham
 * FFT (radix 2/3/4, double); the FP32 Poisson mode rounds to float after each axis.
 * Reference y/z labelling as in mhit_oracle.py (yz_shift).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

typedef struct {
  int nx, ny, nz;
  double dt, mu, rho, f1, f2, f3, k0, radius, sigma, epsr;
  int phiflag, partflag, poisson, laplacian, yz_shift, interp, acdi_clamp;
} orc_params;

typedef struct {
  double re, im;
} cplx;

typedef struct {
  orc_params p;
  size_t n;
  double lx, dx, dxi, ddxi, rhoi, eps, epsi;
  double *u, *v, *w, *ru, *rv, *rw, *pr;
  double *phi, *rphi;
  double *tmp[9]; /* work arrays: rhsu..rhsw, psidi, tanh, normals, fst */
  cplx* spec;     /* (nz, ny, nx/2+1) */
  double *sx, *cx, *sy, *cy, *sz, *cz;
  double *k2x, *k2y, *k2z;
  double* part;
  int np;
  double alpha, beta, gumax;
  long nstep;
} orc_state;

#define IDX(i, j, k) (((size_t)(k) * ny + (j)) * nx + (i))
#define ENUM 1.0e-16

/* ------------------------------------------------------------------ FFT (Stockham) */
static void dft_small(cplx* a, int R, int sign) {
  cplx y[4];
  for (int k = 0; k < R; ++k) {
    double sr = 0, si = 0;
    for (int n = 0; n < R; ++n) {
      double ang = sign * 2.0 * M_PI * (double)((n * k) % R) / R;
      double c = cos(ang), s = sin(ang);
      sr += a[n].re * c - a[n].im * s;
      si += a[n].re * s + a[n].im * c;
    }
    y[k].re = sr;
    y[k].im = si;
  }
  memcpy(a, y, sizeof(cplx) * R);
}

static void butterfly(cplx* a, int R, int sign) {
  if (R == 2) {
    cplx t = a[0];
    a[0].re = t.re + a[1].re; a[0].im = t.im + a[1].im;
    a[1].re = t.re - a[1].re; a[1].im = t.im - a[1].im;
  } else if (R == 4) {
    cplx t0 = {a[0].re + a[2].re, a[0].im + a[2].im};
    cplx t1 = {a[0].re - a[2].re, a[0].im - a[2].im};
    cplx t2 = {a[1].re + a[3].re, a[1].im + a[3].im};
    cplx d = {a[1].re - a[3].re, a[1].im - a[3].im};
    cplx t3 = sign < 0 ? (cplx){d.im, -d.re} : (cplx){-d.im, d.re};
    a[0].re = t0.re + t2.re; a[0].im = t0.im + t2.im;
    a[2].re = t0.re - t2.re; a[2].im = t0.im - t2.im;
    a[1].re = t1.re + t3.re; a[1].im = t1.im + t3.im;
    a[3].re = t1.re - t3.re; a[3].im = t1.im - t3.im;
  } else {
    dft_small(a, R, sign);
  }
}

/* unnormalised transform of x (length n, sign -1 forward / +1 inverse); work has length n */
static void fft1(cplx* x, cplx* work, int n, int sign, const cplx* tw /* exp(-2 pi i m/n) */) {
  cplx* in = x;
  cplx* out = work;
  int p = 1;
  int rem = n;
  while (rem > 1) {
    int R = (rem % 4 == 0) ? 4 : ((rem % 2 == 0) ? 2 : 3);
    int m = n / R;
    for (int t = 0; t < m; ++t) {
      int k = t % p;
      cplx a[4];
      for (int r = 0; r < R; ++r) a[r] = in[t + r * m];
      if (p > 1) {
        for (int r = 1; r < R; ++r) {
          cplx w = tw[(size_t)r * k * (n / (p * R))];
          if (sign > 0) w.im = -w.im;
          double re = a[r].re * w.re - a[r].im * w.im;
          double im = a[r].re * w.im + a[r].im * w.re;
          a[r].re = re;
          a[r].im = im;
        }
      }
      butterfly(a, R, sign);
      int j = (t / p) * p * R + k;
      for (int r = 0; r < R; ++r) out[j + r * p] = a[r];
    }
    cplx* tt = in;
    in = out;
    out = tt;
    p *= R;
    rem /= R;
  }
  if (in != x) memcpy(x, in, sizeof(cplx) * n);
}

static cplx* make_tw(int n) {
  cplx* t = (cplx*)malloc(sizeof(cplx) * n);
  for (int m = 0; m < n; ++m) {
    long double a = 2.0L * 3.141592653589793238462643383279502884L * m / n;
    t[m].re = (double)cosl(a);
    t[m].im = (double)(-sinl(a));
  }
  return t;
}

static inline void round32(cplx* a, int n, int on) {
  if (!on) return;
  for (int i = 0; i < n; ++i) {
    a[i].re = (double)(float)a[i].re;
    a[i].im = (double)(float)a[i].im;
  }
}

/* ------------------------------------------------------------------ setup */
orc_state* orc_create(const orc_params* p) {
  orc_state* s = (orc_state*)calloc(1, sizeof(orc_state));
  s->p = *p;
  int nx = p->nx, ny = p->ny, nz = p->nz;
  s->n = (size_t)nx * ny * nz;
  s->lx = 8.0 * atan(1.0);
  s->dx = s->lx / nx;
  s->dxi = 1.0 / s->dx;
  s->ddxi = 1.0 / s->dx / s->dx;
  s->rhoi = 1.0 / p->rho;
  s->eps = p->epsr * s->dx;
  s->epsi = 1.0 / s->eps;
  size_t b = s->n * sizeof(double);
  s->u = calloc(1, b); s->v = calloc(1, b); s->w = calloc(1, b);
  s->ru = calloc(1, b); s->rv = calloc(1, b); s->rw = calloc(1, b);
  s->pr = calloc(1, b);
  for (int q = 0; q < 9; ++q) s->tmp[q] = calloc(1, b);
  if (p->phiflag) { s->phi = calloc(1, b); s->rphi = calloc(1, b); }
  s->spec = (cplx*)calloc((size_t)(nx / 2 + 1) * ny * nz, sizeof(cplx));
  /* forcing tables: x(i)=x(i-1)+dx accumulated, y/z read one entry on (yz_shift) */
  double* tabs[6];
  int ns[3] = {nx, ny, nz};
  for (int ax = 0; ax < 3; ++ax) {
    int nn = ns[ax];
    double* xc = (double*)malloc(sizeof(double) * (nn + 1));
    double acc = 0.0;
    xc[0] = 0.0;
    for (int i = 1; i <= nn; ++i) { acc = acc + s->dx; xc[i] = acc; }
    int off = ax == 0 ? 0 : p->yz_shift;
    tabs[2 * ax] = (double*)malloc(sizeof(double) * nn);
    tabs[2 * ax + 1] = (double*)malloc(sizeof(double) * nn);
    for (int i = 0; i < nn; ++i) {
      tabs[2 * ax][i] = sin(p->k0 * xc[i + off] + s->dx / 2);
      tabs[2 * ax + 1][i] = cos(p->k0 * xc[i + off] + s->dx / 2);
    }
    free(xc);
  }
  s->sx = tabs[0]; s->cx = tabs[1]; s->sy = tabs[2]; s->cy = tabs[3]; s->sz = tabs[4]; s->cz = tabs[5];
  int lens[3] = {nx / 2 + 1, ny, nz};
  double** k2s[3] = {&s->k2x, &s->k2y, &s->k2z};
  for (int ax = 0; ax < 3; ++ax) {
    int nn = ns[ax], len = lens[ax];
    double* t = (double*)malloc(sizeof(double) * len);
    for (int i = 0; i < len; ++i) {
      double kk = (i < nn / 2) ? (double)i : (double)(i - nn);
      t[i] = p->laplacian ? (2.0 - 2.0 * cos(kk * s->dx)) * s->ddxi : kk * kk;
    }
    *k2s[ax] = t;
  }
  s->alpha = 1.0;
  s->beta = 0.0;
  s->gumax = 1.0;
  return s;
}

void orc_destroy(orc_state* s) {
  if (!s) return;
  free(s->u); free(s->v); free(s->w); free(s->ru); free(s->rv); free(s->rw); free(s->pr);
  for (int q = 0; q < 9; ++q) free(s->tmp[q]);
  free(s->phi); free(s->rphi); free(s->spec);
  free(s->sx); free(s->cx); free(s->sy); free(s->cy); free(s->sz); free(s->cz);
  free(s->k2x); free(s->k2y); free(s->k2z); free(s->part);
  free(s);
}

void orc_set_fields(orc_state* s, const double* u, const double* v, const double* w, const double* phi) {
  size_t b = s->n * sizeof(double);
  memcpy(s->u, u, b); memcpy(s->v, v, b); memcpy(s->w, w, b);
  if (s->p.phiflag && phi) memcpy(s->phi, phi, b);
  memset(s->ru, 0, b); memset(s->rv, 0, b); memset(s->rw, 0, b);
  if (s->rphi) memset(s->rphi, 0, b);
  s->alpha = 1.0; s->beta = 0.0; s->gumax = 1.0; s->nstep = 0;
}

void orc_set_particles(orc_state* s, const double* part, int np) {
  free(s->part);
  s->np = np;
  s->part = (double*)malloc(sizeof(double) * 12 * (size_t)(np > 0 ? np : 1));
  memcpy(s->part, part, sizeof(double) * 12 * (size_t)np);
}

void orc_get_fields(orc_state* s, double* u, double* v, double* w, double* p, double* phi) {
  size_t b = s->n * sizeof(double);
  if (u) memcpy(u, s->u, b);
  if (v) memcpy(v, s->v, b);
  if (w) memcpy(w, s->w, b);
  if (p) memcpy(p, s->pr, b);
  if (phi && s->phi) memcpy(phi, s->phi, b);
}

void orc_get_particles(orc_state* s, double* part) { memcpy(part, s->part, sizeof(double) * 12 * (size_t)s->np); }

double orc_gumax(orc_state* s) { return s->gumax; }

/* ------------------------------------------------------------------ step pieces */
static void tracers(orc_state* s) {
  /* multi/main.f90:477-508, particles.f90:88-119, 364-380 (column-major (np,12)) */
  const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz, np = s->np, sh = s->p.yz_shift;
  const double dx = s->dx, lx = s->lx, dt = s->p.dt, al = s->alpha, be = s->beta;
  double* P = s->part;
#pragma omp parallel for schedule(static)
  for (int q = 0; q < np; ++q) {
    double x = P[1 * (size_t)np + q], y = P[2 * (size_t)np + q], z = P[3 * (size_t)np + q];
    double up, vp, wp;
    if (s->p.interp == 0) {
      double fx = floor(x / dx), fy = floor(y / dx), fz = floor(z / dx);
      double tx = x / dx - fx, ty = y / dx - fy, tz = z / dx - fz;
      long ix = (long)fx, iy = (long)fy - sh, iz = (long)fz - sh;
      int i0 = (int)(((ix % nx) + nx) % nx), i1 = (int)((((ix + 1) % nx) + nx) % nx);
      int j0 = (int)(((iy % ny) + ny) % ny), j1 = (int)((((iy + 1) % ny) + ny) % ny);
      int k0 = (int)(((iz % nz) + nz) % nz), k1 = (int)((((iz + 1) % nz) + nz) % nz);
      up = (1.0 - tx) * s->u[IDX(i0, j0, k0)] + tx * s->u[IDX(i1, j0, k0)];
      vp = (1.0 - ty) * s->v[IDX(i0, j0, k0)] + ty * s->v[IDX(i0, j1, k0)];
      wp = (1.0 - tz) * s->w[IDX(i0, j0, k0)] + tz * s->w[IDX(i0, j0, k1)];
    } else {
      double off[3][3] = {{-0.5, sh, sh}, {0.0, sh - 0.5, sh}, {0.0, sh, sh - 0.5}};
      const double* F[3] = {s->u, s->v, s->w};
      double res[3];
      for (int c = 0; c < 3; ++c) {
        double fx = x / dx - off[c][0], fy = y / dx - off[c][1], fz = z / dx - off[c][2];
        double ix = floor(fx), iy = floor(fy), iz = floor(fz);
        double tx = fx - ix, ty = fy - iy, tz = fz - iz;
        long lx_ = (long)ix, ly = (long)iy, lz = (long)iz;
        int a0 = (int)(((lx_ % nx) + nx) % nx), a1 = (int)((((lx_ + 1) % nx) + nx) % nx);
        int b0 = (int)(((ly % ny) + ny) % ny), b1 = (int)((((ly + 1) % ny) + ny) % ny);
        int c0 = (int)(((lz % nz) + nz) % nz), c1 = (int)((((lz + 1) % nz) + nz) % nz);
        const double* f = F[c];
        double c00 = (1.0 - tx) * f[IDX(a0, b0, c0)] + tx * f[IDX(a1, b0, c0)];
        double c10 = (1.0 - tx) * f[IDX(a0, b1, c0)] + tx * f[IDX(a1, b1, c0)];
        double c01 = (1.0 - tx) * f[IDX(a0, b0, c1)] + tx * f[IDX(a1, b0, c1)];
        double c11 = (1.0 - tx) * f[IDX(a0, b1, c1)] + tx * f[IDX(a1, b1, c1)];
        double d0 = (1.0 - ty) * c00 + ty * c10;
        double d1 = (1.0 - ty) * c01 + ty * c11;
        res[c] = (1.0 - tz) * d0 + tz * d1;
      }
      up = res[0]; vp = res[1]; wp = res[2];
    }
    P[4 * (size_t)np + q] = up; P[5 * (size_t)np + q] = vp; P[6 * (size_t)np + q] = wp;
    x = x + dt * (al * up - be * P[8 * (size_t)np + q]);
    y = y + dt * (al * vp - be * P[9 * (size_t)np + q]);
    z = z + dt * (al * wp - be * P[10 * (size_t)np + q]);
    x = x - lx * floor(x / lx);
    y = y - lx * floor(y / lx);
    z = z - lx * floor(z / lx);
    P[1 * (size_t)np + q] = x; P[2 * (size_t)np + q] = y; P[3 * (size_t)np + q] = z;
    P[8 * (size_t)np + q] = up; P[9 * (size_t)np + q] = vp; P[10 * (size_t)np + q] = wp;
  }
}

#define LOOP3                                             \
  _Pragma("omp parallel for schedule(static) collapse(2)") \
  for (int k = 0; k < nz; ++k)                             \
    for (int j = 0; j < ny; ++j)                           \
      for (int i = 0; i < nx; ++i)

#define NB                                                                  \
  const int ip = i + 1 == nx ? 0 : i + 1, im = i == 0 ? nx - 1 : i - 1;     \
  const int jp = j + 1 == ny ? 0 : j + 1, jm = j == 0 ? ny - 1 : j - 1;     \
  const int kp = k + 1 == nz ? 0 : k + 1, km = k == 0 ? nz - 1 : k - 1;     \
  (void)ip; (void)im; (void)jp; (void)jm; (void)kp; (void)km;

static void phase(orc_state* s) {
  /* multi/main.f90:522-636 */
  const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
  const double eps = s->eps, epsi = s->epsi, dxi = s->dxi, ddxi = s->ddxi;
  double *phi = s->phi, *u = s->u, *v = s->v, *w = s->w;
  double *psi = s->tmp[3], *th = s->tmp[4], *nxa = s->tmp[5], *nya = s->tmp[6], *nza = s->tmp[7];
  double* rhs = s->tmp[8];
  LOOP3 {
    size_t c = IDX(i, j, k);
    double val = fmin(phi[c], 1.0);
    if (s->p.acdi_clamp) val = fmax(val, 0.0);
    psi[c] = eps * log((val + ENUM) / (1.0 - val + ENUM));
    th[c] = tanh(0.5 * psi[c] * epsi);
  }
  const double gamma = 1.0 * s->gumax;
  LOOP3 {
    NB
    size_t c = IDX(i, j, k);
    double p0 = phi[c];
    rhs[c] = -((u[IDX(ip, j, k)] * 0.5 * (phi[IDX(ip, j, k)] + p0) - u[c] * 0.5 * (p0 + phi[IDX(im, j, k)])) * dxi) -
             (v[IDX(i, jp, k)] * 0.5 * (phi[IDX(i, jp, k)] + p0) - v[c] * 0.5 * (p0 + phi[IDX(i, jm, k)])) * dxi -
             (w[IDX(i, j, kp)] * 0.5 * (phi[IDX(i, j, kp)] + p0) - w[c] * 0.5 * (p0 + phi[IDX(i, j, km)])) * dxi +
             gamma * (eps * (phi[IDX(ip, j, k)] - 2.0 * p0 + phi[IDX(im, j, k)]) * ddxi +
                      eps * (phi[IDX(i, jp, k)] - 2.0 * p0 + phi[IDX(i, jm, k)]) * ddxi +
                      eps * (phi[IDX(i, j, kp)] - 2.0 * p0 + phi[IDX(i, j, km)]) * ddxi);
    nxa[c] = psi[IDX(ip, j, k)] - psi[IDX(im, j, k)];
    nya[c] = psi[IDX(i, jp, k)] - psi[IDX(i, jm, k)];
    nza[c] = psi[IDX(i, j, kp)] - psi[IDX(i, j, km)];
  }
  LOOP3 {
    size_t c = IDX(i, j, k);
    double normag = 1.0 / (sqrt(nxa[c] * nxa[c] + nya[c] * nya[c] + nza[c] * nza[c]) + ENUM);
    nxa[c] = nxa[c] * normag;
    nya[c] = nya[c] * normag;
    nza[c] = nza[c] * normag;
  }
  /* F = 0.25 (1 - t^2) n, stored over psi (no longer needed) and th */
  double *fx = psi, *fy = th, *fz = s->tmp[0];
  LOOP3 {
    size_t c = IDX(i, j, k);
    double f = 0.25 * (1.0 - th[c] * th[c]);
    fx[c] = f * nxa[c];
    fz[c] = f * nza[c];
    fy[c] = f * nya[c];
  }
  const double dt = s->p.dt, al = s->alpha, be = s->beta;
  LOOP3 {
    NB
    size_t c = IDX(i, j, k);
    double r = rhs[c] - gamma * ((fx[IDX(ip, j, k)] - fx[IDX(im, j, k)]) * 0.5 * dxi +
                                 (fy[IDX(i, jp, k)] - fy[IDX(i, jm, k)]) * 0.5 * dxi +
                                 (fz[IDX(i, j, kp)] - fz[IDX(i, j, km)]) * 0.5 * dxi);
    rhs[c] = r;
  }
  LOOP3 {
    size_t c = IDX(i, j, k);
    phi[c] = phi[c] + dt * (al * rhs[c] - be * s->rphi[c]);
    s->rphi[c] = rhs[c];
  }
}

static void momentum(orc_state* s) {
  /* multi/main.f90:658-802 */
  const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
  const double dxi = s->dxi, ddxi = s->ddxi, rhoi = s->rhoi, mu = s->p.mu;
  const double f1 = s->p.f1, f2 = s->p.f2, f3 = s->p.f3;
  double *u = s->u, *v = s->v, *w = s->w;
  double *rhsu = s->tmp[0], *rhsv = s->tmp[1], *rhsw = s->tmp[2];
  LOOP3 {
    NB
    size_t c = IDX(i, j, k);
    double h11 = (u[IDX(ip, j, k)] + u[c]) * (u[IDX(ip, j, k)] + u[c]) - (u[c] + u[IDX(im, j, k)]) * (u[c] + u[IDX(im, j, k)]);
    double h12 = (u[IDX(i, jp, k)] + u[c]) * (v[IDX(i, jp, k)] + v[IDX(im, jp, k)]) - (u[c] + u[IDX(i, jm, k)]) * (v[c] + v[IDX(im, j, k)]);
    double h13 = (u[IDX(i, j, kp)] + u[c]) * (w[IDX(i, j, kp)] + w[IDX(im, j, kp)]) - (u[c] + u[IDX(i, j, km)]) * (w[c] + w[IDX(im, j, k)]);
    double h21 = (u[IDX(ip, j, k)] + u[IDX(ip, jm, k)]) * (v[IDX(ip, j, k)] + v[c]) - (u[c] + u[IDX(i, jm, k)]) * (v[c] + v[IDX(im, j, k)]);
    double h22 = (v[IDX(i, jp, k)] + v[c]) * (v[IDX(i, jp, k)] + v[c]) - (v[c] + v[IDX(i, jm, k)]) * (v[c] + v[IDX(i, jm, k)]);
    double h23 = (w[IDX(i, j, kp)] + w[IDX(i, jm, kp)]) * (v[IDX(i, j, kp)] + v[c]) - (w[c] + w[IDX(i, jm, k)]) * (v[c] + v[IDX(i, j, km)]);
    double h31 = (w[IDX(ip, j, k)] + w[c]) * (u[IDX(ip, j, k)] + u[IDX(ip, j, km)]) - (w[c] + w[IDX(im, j, k)]) * (u[c] + u[IDX(i, j, km)]);
    double h32 = (v[IDX(i, jp, k)] + v[IDX(i, jp, km)]) * (w[IDX(i, jp, k)] + w[c]) - (v[c] + v[IDX(i, j, km)]) * (w[c] + w[IDX(i, jm, k)]);
    double h33 = (w[IDX(i, j, kp)] + w[c]) * (w[IDX(i, j, kp)] + w[c]) - (w[c] + w[IDX(i, j, km)]) * (w[c] + w[IDX(i, j, km)]);
    h11 = h11 * 0.25 * dxi; h12 = h12 * 0.25 * dxi; h13 = h13 * 0.25 * dxi;
    h21 = h21 * 0.25 * dxi; h22 = h22 * 0.25 * dxi; h23 = h23 * 0.25 * dxi;
    h31 = h31 * 0.25 * dxi; h32 = h32 * 0.25 * dxi; h33 = h33 * 0.25 * dxi;
    double ru = -(h11 + h12 + h13), rv = -(h21 + h22 + h23), rw = -(h31 + h32 + h33);
    h11 = mu * (u[IDX(ip, j, k)] - 2.0 * u[c] + u[IDX(im, j, k)]) * ddxi;
    h12 = mu * (u[IDX(i, jp, k)] - 2.0 * u[c] + u[IDX(i, jm, k)]) * ddxi;
    h13 = mu * (u[IDX(i, j, kp)] - 2.0 * u[c] + u[IDX(i, j, km)]) * ddxi;
    h21 = mu * (v[IDX(ip, j, k)] - 2.0 * v[c] + v[IDX(im, j, k)]) * ddxi;
    h22 = mu * (v[IDX(i, jp, k)] - 2.0 * v[c] + v[IDX(i, jm, k)]) * ddxi;
    h23 = mu * (v[IDX(i, j, kp)] - 2.0 * v[c] + v[IDX(i, j, km)]) * ddxi;
    h31 = mu * (w[IDX(ip, j, k)] - 2.0 * w[c] + w[IDX(im, j, k)]) * ddxi;
    h32 = mu * (w[IDX(i, jp, k)] - 2.0 * w[c] + w[IDX(i, jm, k)]) * ddxi;
    h33 = mu * (w[IDX(i, j, kp)] - 2.0 * w[c] + w[IDX(i, j, km)]) * ddxi;
    ru = ru + (h11 + h12 + h13) * rhoi;
    rv = rv + (h21 + h22 + h23) * rhoi;
    rw = rw + (h31 + h32 + h33) * rhoi;
    rhsu[c] = ru + f3 * s->sz[k] + f2 * s->cy[j];
    rhsv[c] = rv + f1 * s->sx[i] + f3 * s->cz[k];
    rhsw[c] = rw + f2 * s->sy[j] + f1 * s->cx[i];
  }
  if (s->p.phiflag) {
    /* multi/main.f90:721-780 */
    double *phi = s->phi, *fxs = s->tmp[3], *fys = s->tmp[4], *fzs = s->tmp[5];
    const double eps = s->eps, epsi = s->epsi, sigma = s->p.sigma;
    LOOP3 {
      NB
      size_t c = IDX(i, j, k);
      double p0 = phi[c];
      double chempot = p0 * (1.0 - p0) * (1.0 - 2.0 * p0) * epsi -
                       eps * (phi[IDX(ip, j, k)] + phi[IDX(im, j, k)] + phi[IDX(i, jp, k)] + phi[IDX(i, jm, k)] +
                              phi[IDX(i, j, kp)] + phi[IDX(i, j, km)] - 6.0 * p0) * ddxi;
      fxs[c] = 6.0 * sigma * chempot * 0.5 * (phi[IDX(ip, j, k)] - phi[IDX(im, j, k)]) * dxi;
      fys[c] = 6.0 * sigma * chempot * 0.5 * (phi[IDX(i, jp, k)] - phi[IDX(i, jm, k)]) * dxi;
      fzs[c] = 6.0 * sigma * chempot * 0.5 * (phi[IDX(i, j, kp)] - phi[IDX(i, j, km)]) * dxi;
    }
    LOOP3 {
      NB
      size_t c = IDX(i, j, k);
      rhsu[c] = rhsu[c] + 0.5 * (fxs[IDX(im, j, k)] + fxs[c]) * rhoi;
      rhsv[c] = rhsv[c] + 0.5 * (fys[IDX(i, jm, k)] + fys[c]) * rhoi;
      rhsw[c] = rhsw[c] + 0.5 * (fzs[IDX(i, j, km)] + fzs[c]) * rhoi;
    }
  }
  const double dt = s->p.dt, al = s->alpha, be = s->beta;
  LOOP3 {
    size_t c = IDX(i, j, k);
    u[c] = u[c] + dt * (al * rhsu[c] - be * s->ru[c]);
    v[c] = v[c] + dt * (al * rhsv[c] - be * s->rv[c]);
    w[c] = w[c] + dt * (al * rhsw[c] - be * s->rw[c]);
    s->ru[c] = rhsu[c];
    s->rv[c] = rhsv[c];
    s->rw[c] = rhsw[c];
  }
  s->alpha = 1.5;
  s->beta = 0.5;
}

static void poisson(orc_state* s) {
  /* multi/main.f90:833-923 */
  const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz, nkx = nx / 2 + 1;
  const int f32 = s->p.poisson == 1;
  double *u = s->u, *v = s->v, *w = s->w, *rhsp = s->tmp[0];
  const double cdiv = s->p.rho * s->dxi / s->p.dt;
  LOOP3 {
    NB
    size_t c = IDX(i, j, k);
    double r = cdiv * (u[IDX(ip, j, k)] - u[c]);
    r = r + cdiv * (v[IDX(i, jp, k)] - v[c]);
    r = r + cdiv * (w[IDX(i, j, kp)] - w[c]);
    rhsp[c] = f32 ? (double)(float)r : r;
  }
  cplx *twx = make_tw(nx), *twy = make_tw(ny), *twz = make_tw(nz);
  cplx* S = s->spec;
  int nmax = nx > ny ? nx : ny;
  nmax = nmax > nz ? nmax : nz;
  /* x: R2C by a full complex transform of each line */
#pragma omp parallel
  {
    cplx* a = (cplx*)malloc(sizeof(cplx) * nmax);
    cplx* wk = (cplx*)malloc(sizeof(cplx) * nmax);
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        for (int i = 0; i < nx; ++i) { a[i].re = rhsp[IDX(i, j, k)]; a[i].im = 0.0; }
        fft1(a, wk, nx, -1, twx);
        round32(a, nkx, f32);
        memcpy(S + ((size_t)k * ny + j) * nkx, a, sizeof(cplx) * nkx);
      }
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nkx; ++i) {
        for (int j = 0; j < ny; ++j) a[j] = S[((size_t)k * ny + j) * nkx + i];
        fft1(a, wk, ny, -1, twy);
        round32(a, ny, f32);
        for (int j = 0; j < ny; ++j) S[((size_t)k * ny + j) * nkx + i] = a[j];
      }
    const double ntot = (double)nx * (double)ny * (double)nz;
#pragma omp for collapse(2) schedule(static)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nkx; ++i) {
        for (int k = 0; k < nz; ++k) a[k] = S[((size_t)k * ny + j) * nkx + i];
        fft1(a, wk, nz, -1, twz);
        round32(a, nz, f32);
        for (int k = 0; k < nz; ++k) {
          double k2 = (s->k2x[i] + s->k2y[j]) + s->k2z[k];
          a[k].re = (-a[k].re) / k2 / ntot;
          a[k].im = (-a[k].im) / k2 / ntot;
          if (i == 0 && j == 0 && k == 0) { a[k].re = 0.0; a[k].im = 0.0; }
        }
        round32(a, nz, f32);
        fft1(a, wk, nz, +1, twz);
        round32(a, nz, f32);
        for (int k = 0; k < nz; ++k) S[((size_t)k * ny + j) * nkx + i] = a[k];
      }
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int i = 0; i < nkx; ++i) {
        for (int j = 0; j < ny; ++j) a[j] = S[((size_t)k * ny + j) * nkx + i];
        fft1(a, wk, ny, +1, twy);
        round32(a, ny, f32);
        for (int j = 0; j < ny; ++j) S[((size_t)k * ny + j) * nkx + i] = a[j];
      }
    /* x: C2R from the half spectrum (Hermitian extension, imag of DC/Nyquist dropped) */
#pragma omp for collapse(2) schedule(static)
    for (int k = 0; k < nz; ++k)
      for (int j = 0; j < ny; ++j) {
        const cplx* h = S + ((size_t)k * ny + j) * nkx;
        for (int i = 0; i < nkx; ++i) a[i] = h[i];
        a[0].im = 0.0;
        a[nx / 2].im = 0.0;
        for (int i = nkx; i < nx; ++i) { a[i].re = h[nx - i].re; a[i].im = -h[nx - i].im; }
        fft1(a, wk, nx, +1, twx);
        for (int i = 0; i < nx; ++i) s->pr[IDX(i, j, k)] = f32 ? (double)(float)a[i].re : a[i].re;
      }
    free(a);
    free(wk);
  }
  free(twx); free(twy); free(twz);
}

static void correct(orc_state* s) {
  /* multi/main.f90:942-1003 */
  const int nx = s->p.nx, ny = s->p.ny, nz = s->p.nz;
  double *u = s->u, *v = s->v, *w = s->w, *pr = s->pr;
  const double cc = s->p.dt / s->p.rho, dxi = s->dxi;
  double su = 0, sv = 0, sw = 0;
#pragma omp parallel for schedule(static) collapse(2) reduction(+ : su, sv, sw)
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        NB
        size_t c = IDX(i, j, k);
        u[c] = u[c] - cc * (pr[c] - pr[IDX(im, j, k)]) * dxi;
        v[c] = v[c] - cc * (pr[c] - pr[IDX(i, jm, k)]) * dxi;
        w[c] = w[c] - cc * (pr[c] - pr[IDX(i, j, km)]) * dxi;
        su += u[c];
        sv += v[c];
        sw += w[c];
      }
  double mu = su / nx / ny / nz, mv = sv / nx / ny / nz, mw = sw / nx / ny / nz;
  double uc = -INFINITY, vc = -INFINITY, wc = -INFINITY;
#pragma omp parallel for schedule(static) reduction(max : uc, vc, wc)
  for (size_t c = 0; c < s->n; ++c) {
    u[c] = u[c] - mu;
    v[c] = v[c] - mv;
    w[c] = w[c] - mw;
    uc = fmax(uc, u[c]);
    vc = fmax(vc, v[c]);
    wc = fmax(wc, w[c]);
  }
  s->gumax = fmax(wc, fmax(uc, vc));
}

void orc_step(orc_state* s, int nsteps) {
  for (int t = 0; t < nsteps; ++t) {
    if (s->p.partflag && s->np > 0) tracers(s);
    if (s->p.phiflag) phase(s);
    momentum(s);
    poisson(s);
    correct(s);
    s->nstep++;
  }
}

int orc_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
