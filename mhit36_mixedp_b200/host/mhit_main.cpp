// Host driver in C++ over the C ABI of libmhit_b200.so: the run control of the reference's
// `program main` (multi/main.f90) on one GPU, for hosts without a Fortran compiler.
//
//   input.inp          read by mhit_read_input (subroutine readinput, multi/readinput.f90:4-81)
//   initial condition  inflow = 0: Taylor-Green on the staggered grid (multi/main.f90:322-337),
//                      built on the device by mhit_init_taylor_green;
//                      inflow = 1: u, v, w from <indir>/{u,v,w}.dat (readfield, :339-350);
//                      phiflag: inphi = 0 a centred drop (:370-382, mhit_init_drops with one
//                      centre at (pi, pi, pi)), inphi = 1 <indir>/phi.dat
//   time loop          do t = tstart+1, tfin: one mhit_step per step (:456-1007), the CFL print
//                      of :1003-1007 and its stop at CFL > 7 (:1006), field files every `dump`
//                      steps (:1023-1034, writefield of multi/readwrite.f90)
//
// Fields read from files are uploaded with mhit_upload_fields; a mixed start (velocity from
// files, centred drop) uploads the files first and then builds phi on the device.
#include <sys/stat.h>

#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/mhit_b200.h"

namespace {

struct Options {
  std::string input, indir = "input", outdir;
  int n = 64, ny = 0, nz = 0, steps = -1, phiflag = 0, device = 0;
  int poisson = MHIT_POISSON_FP64, laplacian = MHIT_LAP_EXACT;
  double dt = 0.0;
  bool quiet = false, dry_run = false;
};

void usage() {
  std::printf(
      "usage: mhit_main [--input input.inp] [--n N] [--ny N] [--nz N] [--steps S] [--phiflag 0|1]\n"
      "                 [--poisson fp64|fp32|fp32_refined|fp32_incremental] [--laplacian exact|modified] [--dt DT]\n"
      "                 [--indir DIR] [--outdir DIR] [--device D] [--quiet] [--dry-run]\n"
      "Runs tfin - tstart steps of the MHIT36 loop (multi/main.f90) on one GPU; --dry-run prints the\n"
      "parameters read from input.inp and exits without touching the GPU.\n");
}

bool parse(int argc, char** argv, Options& o) {
  for (int i = 1; i < argc; ++i) {
    const std::string a = argv[i];
    auto val = [&](const char* name) -> const char* {
      if (i + 1 >= argc) {
        std::fprintf(stderr, "missing value after %s\n", name);
        std::exit(2);
      }
      return argv[++i];
    };
    if (a == "--help" || a == "-h") {
      usage();
      std::exit(0);
    } else if (a == "--input") {
      o.input = val("--input");
    } else if (a == "--n") {
      o.n = std::atoi(val("--n"));
    } else if (a == "--ny") {
      o.ny = std::atoi(val("--ny"));
    } else if (a == "--nz") {
      o.nz = std::atoi(val("--nz"));
    } else if (a == "--steps") {
      o.steps = std::atoi(val("--steps"));
    } else if (a == "--phiflag") {
      o.phiflag = std::atoi(val("--phiflag"));
    } else if (a == "--device") {
      o.device = std::atoi(val("--device"));
    } else if (a == "--dt") {
      o.dt = std::atof(val("--dt"));
    } else if (a == "--indir") {
      o.indir = val("--indir");
    } else if (a == "--outdir") {
      o.outdir = val("--outdir");
    } else if (a == "--poisson") {
      const std::string v = val("--poisson");
      if (v == "fp64") o.poisson = MHIT_POISSON_FP64;
      else if (v == "fp32") o.poisson = MHIT_POISSON_FP32;
      else if (v == "fp32_refined") o.poisson = MHIT_POISSON_FP32_REFINED;
      else if (v == "fp32_incremental") o.poisson = MHIT_POISSON_FP32_INCREMENTAL;
      else return false;
    } else if (a == "--laplacian") {
      const std::string v = val("--laplacian");
      if (v == "exact") o.laplacian = MHIT_LAP_EXACT;
      else if (v == "modified") o.laplacian = MHIT_LAP_MODIFIED;
      else return false;
    } else if (a == "--quiet") {
      o.quiet = true;
    } else if (a == "--dry-run") {
      o.dry_run = true;
    } else {
      std::fprintf(stderr, "unknown option %s\n", a.c_str());
      return false;
    }
  }
  return o.n > 0;
}

int fail(const char* what, int rc) {
  std::fprintf(stderr, "%s failed (%d): %s\n", what, rc, mhit_last_error());
  return 1;
}

bool read_raw(const std::string& path, std::vector<double>& a) {
  FILE* f = std::fopen(path.c_str(), "rb");
  if (!f) return false;
  const size_t got = std::fread(a.data(), sizeof(double), a.size(), f);
  std::fclose(f);
  return got == a.size();
}

}  // namespace

int main(int argc, char** argv) {
  Options o;
  if (!parse(argc, argv, o)) {
    usage();
    return 2;
  }
  mhit_params p;
  int rc = mhit_params_default(&p);
  if (rc) return fail("mhit_params_default", rc);
  p.nx = o.n;
  p.ny = o.ny ? o.ny : o.n;
  p.nz = o.nz ? o.nz : o.n;
  p.phiflag = o.phiflag;
  p.poisson = o.poisson;
  p.laplacian = o.laplacian;
  p.device = o.device;
  mhit_run run = {0, 0, 10, 1000000000, 0, 0, 0};
  if (!o.input.empty() && (rc = mhit_read_input(o.input.c_str(), &p, &run))) return fail("mhit_read_input", rc);
  if (o.dt > 0.0) p.dt = o.dt;
  const int steps = o.steps >= 0 ? o.steps : run.tfin - run.tstart;
  if (o.dry_run) {
    std::printf(
        "{\"nx\": %d, \"ny\": %d, \"nz\": %d, \"dt\": %.17g, \"mu\": %.17g, \"rho\": %.17g, \"f1\": %.17g, "
        "\"f2\": %.17g, \"f3\": %.17g, \"k0\": %.17g, \"radius\": %.17g, \"sigma\": %.17g, \"epsr\": %.17g, "
        "\"npart\": %d, \"restart\": %d, \"tstart\": %d, \"tfin\": %d, \"dump\": %d, \"inflow\": %d, \"inphi\": %d, "
        "\"inpart\": %d, \"steps\": %d}\n",
        p.nx, p.ny, p.nz, p.dt, p.mu, p.rho, p.f1, p.f2, p.f3, p.k0, p.radius, p.sigma, p.epsr, p.npart, run.restart,
        run.tstart, run.tfin, run.dump, run.inflow, run.inphi, run.inpart, steps);
    return 0;
  }

  const size_t n = (size_t)p.nx * p.ny * p.nz;
  mhit_ctx* ctx = nullptr;
  if ((rc = mhit_init(&p, &ctx))) return fail("mhit_init", rc);
  auto bail = [&](const char* what, int r) {
    mhit_destroy(ctx);
    return fail(what, r);
  };
  if (run.inflow == 1) {
    std::vector<double> u(n), v(n), w(n), phi(p.phiflag ? n : 0);
    for (auto [name, a] : {std::pair<const char*, std::vector<double>*>{"u", &u}, {"v", &v}, {"w", &w}}) {
      const std::string path = o.indir + "/" + name + ".dat";
      if (!read_raw(path, *a)) {
        std::fprintf(stderr, "cannot read %s\n", path.c_str());
        mhit_destroy(ctx);
        return 1;
      }
    }
    // phi from the file when inphi = 1; otherwise a placeholder replaced by the drop below
    if (p.phiflag && run.inphi == 1 && !read_raw(o.indir + "/phi.dat", phi)) {
      std::fprintf(stderr, "cannot read %s/phi.dat\n", o.indir.c_str());
      mhit_destroy(ctx);
      return 1;
    }
    if ((rc = mhit_upload_fields(ctx, u.data(), v.data(), w.data(), p.phiflag ? phi.data() : nullptr)))
      return bail("mhit_upload_fields", rc);
  } else {
    if ((rc = mhit_init_taylor_green(ctx))) return bail("mhit_init_taylor_green", rc);
    if (p.phiflag && run.inphi == 1) {
      if ((rc = mhit_read_field(ctx, (o.indir + "/phi.dat").c_str(), 5))) return bail("mhit_read_field", rc);
    }
  }
  if (p.phiflag && run.inphi != 1) {
    const double pi = 4.0 * std::atan(1.0);
    const double centre[3] = {pi, pi, pi};
    if ((rc = mhit_init_drops(ctx, 1, centre, p.radius))) return bail("mhit_init_drops", rc);
  }
  const int nfields = p.phiflag ? 5 : 4;
  auto dump = [&](int t) -> int {
    for (int f = 1; f <= nfields; ++f) {
      const int r = mhit_write_field(ctx, o.outdir.c_str(), t, f);
      if (r) return fail("mhit_write_field", r);
    }
    return 0;
  };
  if (!o.outdir.empty()) {
    mkdir(o.outdir.c_str(), 0755);
    if (dump(run.tstart)) {
      mhit_destroy(ctx);
      return 1;
    }
  }
  const auto t0 = std::chrono::steady_clock::now();
  int status = 0;
  mhit_diag d;
  for (int t = run.tstart + 1; t <= run.tstart + steps; ++t) {
    rc = mhit_step(ctx, 1);
    if (rc == MHIT_ERR_CFL) {  // multi/main.f90:1006
      std::printf("CFL > 7 at step %d: stop\n", t);
      status = 3;
      break;
    }
    if (rc) {
      status = fail("mhit_step", rc);
      break;
    }
    if (!o.quiet && (rc = mhit_diagnostics(ctx, &d)) == 0)  // the per-step print of :1003-1007
      std::printf("step %d  gumax %.6e  CFL %.6e\n", t, d.gumax, d.cfl);
    if (!o.outdir.empty() && t % run.dump == 0 && dump(t)) {
      status = 1;
      break;
    }
  }
  const double wall = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  if (status == 0 && (rc = mhit_diagnostics(ctx, &d)) == 0)
    std::printf(
        "{\"steps\": %d, \"wall_s\": %.6f, \"ms_per_step\": %.6f, \"nstep\": %lld, \"gumax\": %.17g, \"cfl\": %.17g, "
        "\"maxdiv\": %.17g, \"ke\": %.17g, \"dissipation\": %.17g, \"flags\": %d}\n",
        steps, wall, 1e3 * wall / (steps > 0 ? steps : 1), d.nstep, d.gumax, d.cfl, d.maxdiv, d.ke, d.dissipation,
        d.flags);
  mhit_destroy(ctx);
  return status;
}
