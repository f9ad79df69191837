// Drop-in driver for the single-rank job of the reference (bin/a.out, main.cu:123-580):
// reads params.json (argv[1] or ./params.json), the Fault_geometry / Fault_init_stress
// NetCDF files and the Media1D table, runs NT steps and writes the reference's NetCDF
// outputs into OUT every EXPORT_TIME_SKIP steps (before the step, main.cu:425-437).
#include <sys/time.h>

#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "../../include/dfd_b200.h"
#include "dfd_host.h"

static double now() {
  struct timeval tv;
  gettimeofday(&tv, nullptr);
  return tv.tv_sec + 1e-6 * tv.tv_usec;
}

int main(int argc, char** argv) {
  const char* path = argc > 1 ? argv[1] : "params.json";
  dfd_params p;
  int r = dfd_params_load_json(path, &p);
  if (r) { fprintf(stderr, "cannot read %s: %s\n", path, dfd_error_string(r)); return 1; }
  dfd_ctx* ctx = nullptr;
  r = dfd_create(&p, 0, &ctx);
  if (r) { fprintf(stderr, "dfd_create: %s\n", dfd_error_string(r)); return 1; }
  long nf = (long)p.NY * p.NZ;
  std::string err;
  if (p.INPORT_GRID_TYPE == 1) {
    std::vector<float> g(3 * nf);
    const char* v[3] = {"x", "y", "z"};
    for (int c = 0; c < 3; c++)
      if (!dfd::nc_read_plane(p.Fault_geometry, v[c], p.NZ, p.NY, g.data() + c * nf, &err)) {
        fprintf(stderr, "%s\n", err.c_str());
        return 1;
      }
    dfd_load_fault_geometry(ctx, g.data());
  }
  if (p.INPORT_STRESS_TYPE == 1) {
    std::vector<float> s(15 * nf, 0.0f);
    const char* v[15] = {"Tx", "Ty", "Tz", "dTx", "dTy", "dTz", "mu_s", "mu_d", "Dc", "C0", "a", "b", "L", "Vw",
                         "State"};
    int lo = p.Friction_type == 0 ? 0 : 0, n = 15;
    for (int c = lo; c < n; c++) {
      bool need = c < 6 || (p.Friction_type == 0 ? c < 10 : c >= 10);
      if (!dfd::nc_read_plane(p.Fault_init_stress, v[c], p.NZ, p.NY, s.data() + c * nf, &err) && need) {
        fprintf(stderr, "%s\n", err.c_str());
        return 1;
      }
    }
    dfd_load_fault_init(ctx, s.data());
    if (p.Friction_type == 3) {
      // hydraulic diffusivity of the thermal pressurisation (init.cu:999-1003)
      std::vector<float> hy(nf);
      if (!dfd::nc_read_plane(p.Fault_init_stress, "TP_hy", p.NZ, p.NY, hy.data(), &err)) {
        fprintf(stderr, "%s\n", err.c_str());
        return 1;
      }
      dfd_load_tp_hy(ctx, hy.data());
    }
  }
  if (p.Media1D[0]) {
    FILE* f = fopen(p.Media1D, "r");
    if (!f) { fprintf(stderr, "can not open input media dat\n"); return 1; }
    char line[1024];
    int n = 0;
    if (!fgets(line, sizeof line, f) || fscanf(f, "%d\n", &n) != 1 || !fgets(line, sizeof line, f)) return 1;
    std::vector<float> lay(4 * n);
    for (int i = 0; i < n; i++)
      if (fscanf(f, "%g %g %g %g", &lay[4 * i], &lay[4 * i + 1], &lay[4 * i + 2], &lay[4 * i + 3]) != 4) return 1;
    fclose(f);
    dfd_load_media1d(ctx, n, lay.data());
  }
  r = dfd_precompute(ctx);
  if (r) { fprintf(stderr, "setup: %s (%s)\n", dfd_error_string(r), dfd_last_error(ctx)); return 1; }
  r = dfd_output_open(ctx, p.OUT);
  if (r) { fprintf(stderr, "output: %s\n", dfd_last_error(ctx)); return 1; }
  double total = 0;
  for (int it = 0; it < p.NT; it++) {
    double t0 = now();
    if (it % p.EXPORT_TIME_SKIP == 0) dfd_output_write(ctx, it / p.EXPORT_TIME_SKIP);
    r = dfd_step(ctx, it);
    if (!r) r = dfd_synchronize(ctx);
    if (r) { fprintf(stderr, "step %d: %s (%s)\n", it, dfd_error_string(r), dfd_last_error(ctx)); return 1; }
    double dt = now() - t0;
    total += dt;
    if (it % 10 == 0) { printf("> %6d, total %d, %8.4f s\n", it, p.NT, dt); fflush(stdout); }
  }
  dfd_output_close(ctx);
  printf("----------------------------------\n> Total %6d: %e s\n", p.NT, total);
  dfd_destroy(ctx);
  return 0;
}
