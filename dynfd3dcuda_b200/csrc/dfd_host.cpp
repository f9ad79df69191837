// Host-side pieces of the B200 dynamic-rupture step: job parameters (the reference's
// params.json keys, set_params.cu:56-297), PML and Cerjan 1-D profiles, the separable grid
// description and the on-fault initial state.
#include "dfd_host.h"

#include <cctype>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <vector>

namespace dfd {

// ------------------------------------------------------------------ JSON ----
// A small JSON reader sufficient for job files: objects, arrays, numbers, strings,
// true/false/null.  Values are kept as text and converted on lookup.
struct JVal {
  enum Kind { NUL, NUM, STR, ARR, OBJ, BOOL } kind = NUL;
  double num = 0;
  std::string str;
  std::vector<JVal> arr;
  std::vector<std::pair<std::string, JVal>> obj;
};

struct JParser {
  const char* s;
  bool ok = true;
  void ws() { while (*s && isspace((unsigned char)*s)) s++; }
  bool parse(JVal& v) {
    ws();
    if (*s == '{') {
      v.kind = JVal::OBJ;
      s++;
      ws();
      if (*s == '}') { s++; return true; }
      while (true) {
        ws();
        JVal key;
        if (*s != '"' || !parse(key)) return ok = false;
        ws();
        if (*s != ':') return ok = false;
        s++;
        JVal val;
        if (!parse(val)) return ok = false;
        v.obj.emplace_back(key.str, val);
        ws();
        if (*s == ',') { s++; continue; }
        if (*s == '}') { s++; return true; }
        return ok = false;
      }
    }
    if (*s == '[') {
      v.kind = JVal::ARR;
      s++;
      ws();
      if (*s == ']') { s++; return true; }
      while (true) {
        JVal e;
        if (!parse(e)) return ok = false;
        v.arr.push_back(e);
        ws();
        if (*s == ',') { s++; continue; }
        if (*s == ']') { s++; return true; }
        return ok = false;
      }
    }
    if (*s == '"') {
      v.kind = JVal::STR;
      s++;
      while (*s && *s != '"') {
        if (*s == '\\' && s[1]) {
          s++;
          char c = *s == 'n' ? '\n' : *s == 't' ? '\t' : *s;
          v.str.push_back(c);
          s++;
        } else {
          v.str.push_back(*s++);
        }
      }
      if (*s != '"') return ok = false;
      s++;
      return true;
    }
    if (!strncmp(s, "true", 4)) { v.kind = JVal::BOOL; v.num = 1; s += 4; return true; }
    if (!strncmp(s, "false", 5)) { v.kind = JVal::BOOL; v.num = 0; s += 5; return true; }
    if (!strncmp(s, "null", 4)) { v.kind = JVal::NUL; s += 4; return true; }
    char* end = nullptr;
    double d = strtod(s, &end);
    if (end == s) return ok = false;
    v.kind = JVal::NUM;
    v.num = d;
    s = end;
    return true;
  }
};

void params_default(dfd_params* p) {
  memset(p, 0, sizeof(*p));
  // set_params.cu:60-103, with the PML defaults of :263-267
  strcpy(p->OUT, "output");
  strcpy(p->Fault_geometry, "Fault_geometry.nc");
  strcpy(p->Fault_init_stress, "Fault_init_stress.nc");
  p->EXPORT_TIME_SKIP = 1;
  p->TMAX = 1.0; p->DT = 0.01; p->DH = 100.0;
  p->NX = 100; p->NY = 90; p->NZ = 80;
  p->mu_s = 0.677; p->mu_d = 0.525; p->Dc = 0.4; p->C0 = 0.0;
  p->PML_N = 20; p->PML_velocity = 3000.0; p->PML_bmax = 3.0; p->PML_fc = 1.0;
  p->DAMP_N = 20;
  p->bi_vp1 = 6000.0; p->bi_vs1 = 3464.0; p->bi_rho1 = 2670.0;
  p->bi_vp2 = 6000.0; p->bi_vs2 = 3464.0; p->bi_rho2 = 2670.0;
  // reference Makefile default switches (Makefile:57-161)
  p->rupture = 1; p->free_surface = 1; p->use_pml = 1; p->use_cerjan = 0; p->normal_refine = 1;
  p->rs_guess = 0;
  p->TP_n = 1;  // set_params.cu:103
  p->rs_guess_tol = 1e-10;
  p->slabs_y = 1;
  p->slab_y = 0;
  finalize_params(p);
}

void finalize_params(dfd_params* p) {
  // set_params.cu:286-295 (NT truncates; jobs carry TMAX + DT/2)
  p->NT = (int)((float)p->TMAX / (float)p->DT);
}

int params_from_json(const char* text, dfd_params* p, std::string* err) {
  JParser ps{text};
  JVal root;
  if (!ps.parse(root) || root.kind != JVal::OBJ) {
    if (err) *err = "malformed JSON";
    return DFD_ERR_IO;
  }
  for (auto& kv : root.obj) {
    const std::string& k = kv.first;
    const JVal& v = kv.second;
    auto num = [&](double& dst) { if (v.kind == JVal::NUM || v.kind == JVal::BOOL) dst = v.num; };
    auto inum = [&](int& dst) { if (v.kind == JVal::NUM || v.kind == JVal::BOOL) dst = (int)v.num; };
    auto str = [&](char* dst) {
      if (v.kind == JVal::STR) { strncpy(dst, v.str.c_str(), 1023); dst[1023] = 0; }
    };
    auto arr4 = [&](int* dst) {
      if (v.kind == JVal::ARR)
        for (size_t i = 0; i < 4 && i < v.arr.size(); i++) dst[i] = (int)v.arr[i].num;
    };
    if (k == "OUT") str(p->OUT);
    else if (k == "Fault_geometry") str(p->Fault_geometry);
    else if (k == "Fault_init_stress") str(p->Fault_init_stress);
    else if (k == "Media1D") str(p->Media1D);
    else if (k == "Fault_grid") arr4(p->Fault_grid);
    else if (k == "Asp_grid") arr4(p->Asp_grid);
    else if (k == "TMAX") num(p->TMAX);
    else if (k == "DT") num(p->DT);
    else if (k == "DH") num(p->DH);
    else if (k == "NX") inum(p->NX);
    else if (k == "NY") inum(p->NY);
    else if (k == "NZ") inum(p->NZ);
    else if (k == "viscosity") num(p->viscosity);
    else if (k == "INPORT_GRID_TYPE") inum(p->INPORT_GRID_TYPE);
    else if (k == "INPORT_STRESS_TYPE") inum(p->INPORT_STRESS_TYPE);
    else if (k == "EXPORT_TIME_SKIP") inum(p->EXPORT_TIME_SKIP);
    else if (k == "EXPORT_WAVE_SLICE_X") inum(p->EXPORT_WAVE_SLICE_X);
    else if (k == "EXPORT_WAVE_SLICE_Y") inum(p->EXPORT_WAVE_SLICE_Y);
    else if (k == "EXPORT_WAVE_SLICE_Z") inum(p->EXPORT_WAVE_SLICE_Z);
    else if (k == "Friction_type") inum(p->Friction_type);
    else if (k == "mu_s") num(p->mu_s);
    else if (k == "mu_0") num(p->mu_0);
    else if (k == "mu_d") num(p->mu_d);
    else if (k == "Dc") num(p->Dc);
    else if (k == "C0") num(p->C0);
    else if (k == "RS_V0") num(p->V0);
    else if (k == "RS_Vini") num(p->Vini);
    else if (k == "RS_f0") num(p->f0);
    else if (k == "RS_fw") num(p->fw);
    else if (k == "RS_L") num(p->L);
    else if (k == "smooth_load_T") num(p->smooth_load_T);
    else if (k == "rho1" || k == "bi_rho1") num(p->bi_rho1);  // "rho1" lands in bi_rho1 (set_params.cu:247)
    else if (k == "bi_vs1") num(p->bi_vs1);
    else if (k == "bi_vp1") num(p->bi_vp1);
    else if (k == "bi_vs2") num(p->bi_vs2);
    else if (k == "bi_vp2") num(p->bi_vp2);
    else if (k == "bi_rho2") num(p->bi_rho2);
    else if (k == "PML_N") inum(p->PML_N);
    else if (k == "PML_velocity") num(p->PML_velocity);
    else if (k == "PML_bmax") num(p->PML_bmax);
    else if (k == "PML_fc") num(p->PML_fc);
    else if (k == "DAMP_N") inum(p->DAMP_N);
    // reference compile-time switches, accepted as job keys
    else if (k == "Rupture") inum(p->rupture);
    else if (k == "FreeSurface") inum(p->free_surface);
    else if (k == "usePML") inum(p->use_pml);
    else if (k == "useCerjan") inum(p->use_cerjan);
    else if (k == "NormalRefine") inum(p->normal_refine);
    else if (k == "RS_guess") inum(p->rs_guess);
    else if (k == "RS_guess_tol") num(p->rs_guess_tol);
    else if (k == "TP_n") inum(p->TP_n);  // set_params.cu:281-282
    // PX/PY/PZ, igpu, vp1/vs1, RupThres, smoothing keys: accepted, not used on one GPU
  }
  finalize_params(p);
  return DFD_OK;
}

int check_params(const dfd_params* p, std::string* err) {
  auto fail = [&](const char* m) { if (err) *err = m; return DFD_ERR_PARAM; };
  if (p->NX < 8 || p->NY < 8 || p->NZ < 8) return fail("NX, NY, NZ must be >= 8");
  if (!(p->DT > 0) || !(p->DH > 0)) return fail("DT and DH must be positive");
  if (p->Friction_type < 0 || p->Friction_type > 3)
    return fail("Friction_type must be 0 (slip weakening), 1 (aging law), 2 (slip law) or 3 (slip law with "
                "thermal pressurisation)");
  // the column spacing is width / (TP_n - 1): at the reference's default TP_n = 1 it is
  // infinite and the heat source at the fault, exp(-(0 * inf)^2 ...), is NaN
  // (thermpress.cu:167-196)
  if (p->rupture && p->Friction_type == 3 && (p->TP_n < 2 || p->TP_n > 4096))
    return fail("Friction_type 3 needs 2 <= TP_n <= 4096 points per thermal-pressurisation column");
  if (p->use_pml && (p->PML_N < 2 || 2 * p->PML_N > p->NX || 2 * p->PML_N > p->NY || p->PML_N > p->NZ))
    return fail("PML_N out of range for the grid");
  if (p->use_pml && p->PML_N > 30)
    return fail("PML_N > 30 overlaps the fault band (non-united fault nodes start 31 nodes in)");
  if (p->use_cerjan && (2 * p->DAMP_N > p->NX || 2 * p->DAMP_N > p->NY || 2 * p->DAMP_N > p->NZ))
    return fail("DAMP_N too large for the grid");
  if (!(p->rs_guess_tol >= 0.0 && p->rs_guess_tol < 1.0)) return fail("RS_guess_tol must lie in [0, 1)");
  if (p->EXPORT_TIME_SKIP < 1) return fail("EXPORT_TIME_SKIP must be >= 1");
  // decomposition along y: equal slabs (the reference's nj = NY / PY, set_params.cu), each
  // wide enough for its PML slab and the three-column halo
  if (p->slabs_y < 1 || p->slab_y < 0 || p->slab_y >= p->slabs_y) return fail("slabs_y >= 1 and 0 <= slab_y < slabs_y");
  if (p->slabs_y > 1) {
    if (p->NY % p->slabs_y) return fail("NY must be a multiple of slabs_y");
    const int nj = p->NY / p->slabs_y;
    if (nj < 8 || (p->use_pml && nj < p->PML_N + 4) || (p->use_cerjan && nj < p->DAMP_N + 4))
      return fail("NY / slabs_y too small for the PML, the sponge or the halo");
  }
  return DFD_OK;
}

// ADE CFS-PML 1-D profiles (init_pml.cu:18-133): d ~ x^2 with R from N, alpha linear,
// beta quadratic; D stored divided by beta.
void pml_profile(const dfd_params* p, int n, bool lo, bool hi, std::vector<float>& A, std::vector<float>& B,
                 std::vector<float>& D) {
  A.assign(n, 0.0f); B.assign(n, 1.0f); D.assign(n, 0.0f);
  int N = p->PML_N;
  std::vector<double> Lx(n, -1.0);
  if (lo) for (int i = 0; i < N; i++) Lx[i] = (N - 1 - i) * p->DH;
  if (hi) for (int i = 0; i < N; i++) Lx[n - N + i] = i * p->DH;
  double Rpp = pow(10.0, -((log10((double)N) - 1.0) / log10(2.0) + 3.0));
  double amax = M_PI * p->PML_fc;
  double L0 = p->DH * (N - 1);
  double dmax = -p->PML_velocity / (2.0 * L0) * log(Rpp) * 3.0;
  for (int i = 0; i < n; i++) {
    double x = Lx[i];
    if (x < 0) continue;
    double av = amax * (1.0 - x / L0);
    double bv = 1.0 + (p->PML_bmax - 1.0) * (x / L0) * (x / L0);
    double dv = dmax * (x / L0) * (x / L0);
    A[i] = (float)av;
    B[i] = (float)bv;
    D[i] = (float)(dv / bv);
  }
}

// Cerjan sponge factors on the padded index of one axis (cerjan.cu:31-140): the 3-D
// table of the reference is min(dx[i], dy[j], dz[k]) of these profiles when the faces of
// an axis do not overlap.
void cerjan_profile(const dfd_params* p, int npad, bool lo, bool hi, std::vector<float>& out) {
  out.assign(npad, 1.0f);
  int ND = p->DAMP_N;
  float coef = 0.92f;
  float alpha = (float)(sqrt(-log((double)coef)) / ND);
  for (int d = 0; d < ND; d++) {
    float v = expf(-powf(alpha * (ND - d), 2));
    if (lo) out[3 + d] = v;
    if (hi) out[npad - 3 - d - 1] = v;
  }
}

// x line with normal refinement around the fault (coord.cu:173-209) or the uniform
// Cartesian line, then the linear ghost extrapolation (metric.cu:263-280).
void x_line(const dfd_params* p, std::vector<double>& xl) {
  int nx = p->NX + 6;
  xl.assign(nx, 0.0);
  if (p->normal_refine) {
    std::vector<double> x(nx, 0.0);
    int ic = p->NX / 2 + 3;
    const int w1 = 10, w2 = 55;
    for (int i = ic + 1; i < nx; i++) {
      int dist = abs(i - ic);
      double c = dist < w1 ? 0.0 : (dist < w2 ? 1.0 - cos(M_PI * (i - (ic + w1)) / (double)(w2 - w1)) : 2.0);
      x[i] = x[i - 1] + p->DH * (0.5 + 0.25 * c);
    }
    for (int i = ic - 1; i >= 0; i--) {
      int dist = abs(i - ic);
      double c = dist < w1 ? 0.0 : (dist < w2 ? 1.0 - cos(M_PI * (i - (ic - w1)) / (double)(w2 - w1)) : 2.0);
      x[i] = x[i + 1] - p->DH * (0.5 + 0.25 * c);
    }
    xl = x;
  } else {
    double x0 = -(p->NX / 2) * p->DH;
    for (int i = 0; i < nx; i++) xl[i] = (i - 3) * p->DH + x0;
  }
  for (int n = 1; n <= 3; n++) {
    xl[3 - n] = 2.0 * xl[3] - xl[3 + n];
    xl[nx - 4 + n] = 2.0 * xl[nx - 4] - xl[nx - 4 - n];
  }
}

// Fault surface arrays (nz, ny) with ghosts: the loaded geometry (INPORT_GRID_TYPE == 1,
// coord.cu:299-311) or the flat default, extrapolated first along y then along z.
void surface(const dfd_params* p, const float* fxyz, std::vector<double>& fx, std::vector<double>& fy,
             std::vector<double>& fz) {
  int nj = p->NY, nk = p->NZ, ny = nj + 6, nz = nk + 6;
  fx.assign((size_t)ny * nz, 0.0); fy = fx; fz = fx;
  double y0 = -(p->NY / 2) * p->DH, z0 = (1 - p->NZ) * p->DH;
  for (int k = 0; k < nk; k++)
    for (int j = 0; j < nj; j++) {
      size_t f = (j + 3) + (size_t)(k + 3) * ny;
      if (p->INPORT_GRID_TYPE == 1 && fxyz) {
        size_t q = j + (size_t)k * nj, nf = (size_t)nj * nk;
        fx[f] = fxyz[q]; fy[f] = fxyz[nf + q]; fz[f] = fxyz[2 * nf + q];
      } else {
        fx[f] = 0.0; fy[f] = j * p->DH + y0; fz[f] = k * p->DH + z0;
      }
    }
  std::vector<double>* arrs[3] = {&fx, &fy, &fz};
  for (auto* a : arrs) {
    std::vector<double>& A = *a;
    for (int k = 3; k < nz - 3; k++)
      for (int n = 1; n <= 3; n++) {
        A[(3 - n) + (size_t)k * ny] = 2.0 * A[3 + (size_t)k * ny] - A[(3 + n) + (size_t)k * ny];
        A[(ny - 4 + n) + (size_t)k * ny] = 2.0 * A[(ny - 4) + (size_t)k * ny] - A[(ny - 4 - n) + (size_t)k * ny];
      }
    for (int j = 0; j < ny; j++)
      for (int n = 1; n <= 3; n++) {
        A[j + (size_t)(3 - n) * ny] = 2.0 * A[j + (size_t)3 * ny] - A[j + (size_t)(3 + n) * ny];
        A[j + (size_t)(nz - 4 + n) * ny] = 2.0 * A[j + (size_t)(nz - 4) * ny] - A[j + (size_t)(nz - 4 - n) * ny];
      }
  }
}

// On-fault masks and background state (init.cu:160-849) and the loaded stress and
// friction planes (init.cu:904-1005).  vecn/vecs1/vecs2: (3, nz, ny) planes.
void fault_init(const dfd_params* p, const float* planes, const float* vecn, const float* vecs1, const float* vecs2,
                FaultHost& h) {
  // slab slab_y of a domain decomposed along y: local columns j, global columns j0 + j
  // (the masks and the input planes are global, init.cu:779-816 with gj = ranky nj + j)
  const int nj = p->NY / p->slabs_y, j0 = p->slab_y * nj, NYg = p->NY;
  int nk = p->NZ, ny = nj + 6, nz = nk + 6;
  size_t nf = (size_t)nj * nk, nyz = (size_t)ny * nz;
  h.resize(nf);
  bool fs = p->free_surface != 0;
  for (int k = 0; k < nk; k++)
    for (int j = 0; j < nj; j++) {
      size_t q = j + (size_t)k * nj, f = (j + 3) + (size_t)(k + 3) * ny;
      int gj1 = j0 + j + 1, gk1 = k + 1;
      const int* fg = p->Fault_grid;
      h.rupy[q] = (gj1 <= fg[0] + 3 || gj1 >= fg[1] - 3) ? 0 : 1;
      h.rupz[q] = (gk1 <= fg[2] + 3 || gk1 >= fg[3] - 3) ? 0 : 1;
      bool inner = gj1 > 30 && gj1 < NYg - 30 && gk1 > 30 && (fs || gk1 < p->NZ - 30);
      h.united[q] = inner ? 0 : 1;
      h.faultgrid[q] = (gj1 >= fg[0] + 3 && gj1 <= fg[1] - 3 && gk1 >= fg[2] + 3 && gk1 <= fg[3] - 3) ? 1 : 0;
      // rate-and-state runs test a-b before the friction planes are read; the zero-filled
      // allocation makes that test false everywhere (init.cu:833-844 before :904)
      if (p->Friction_type >= 1) h.faultgrid[q] = 0;
      h.str_peak[q] = (gj1 >= fg[0] && gj1 <= fg[1] && gk1 >= fg[2] && gk1 <= fg[3]) ? (float)p->mu_s : 10000.f;
      h.init_t0[q] = -9999.9f;
      double tn = -120.0e6, ts1 = -120.0e6 * p->mu_0, ts2 = 0.0;
      const int* ag = p->Asp_grid;
      if (gj1 >= ag[0] && gj1 <= ag[1] && gk1 >= ag[2] && gk1 <= ag[3])
        ts1 = (p->mu_s + (p->mu_s - p->mu_d) * 0.001) * -120.0e6;
      h.Tn[q] = (float)tn; h.Ts1[q] = (float)ts1; h.Ts2[q] = (float)ts2;
      for (int c = 0; c < 3; c++) {
        double v = tn * vecn[c * nyz + f] + ts1 * vecs1[c * nyz + f] + ts2 * vecs2[c * nyz + f];
        (c == 0 ? h.sx : c == 1 ? h.sy : h.sz)[q] = (float)v;
      }
    }
  if (p->INPORT_STRESS_TYPE == 1 && planes) {
    // global planes (15, NZ, NY): this slab's columns
    const size_t nfg = (size_t)NYg * nk;
    auto pl = [&](int c, size_t q) { return planes[c * nfg + (q % nj) + j0 + (q / nj) * (size_t)NYg]; };
    std::vector<float>* dst[6] = {&h.T0x, &h.T0y, &h.T0z, &h.dT0x, &h.dT0y, &h.dT0z};
    for (int c = 0; c < 6; c++)
      for (size_t q = 0; q < nf; q++) (*dst[c])[q] = pl(c, q);
    if (p->Friction_type == 0) {
      for (size_t q = 0; q < nf; q++) {
        h.str_peak[q] = pl(6, q); h.Dc[q] = pl(8, q); h.C0[q] = pl(9, q);
      }
    } else {
      for (size_t q = 0; q < nf; q++) {
        h.a[q] = pl(10, q); h.b[q] = pl(11, q); h.L[q] = pl(12, q);
        h.Vw[q] = pl(13, q); h.State[q] = pl(14, q);
      }
    }
    // traction of the loaded stress in the local frame (init.cu:859-902)
    for (int k = 0; k < nk; k++)
      for (int j = 0; j < nj; j++) {
        size_t q = j + (size_t)k * nj, f = (j + 3) + (size_t)(k + 3) * ny;
        double T[3] = {h.T0x[q], h.T0y[q], h.T0z[q]};
        h.Tn[q] = (float)(T[0] * vecn[f] + T[1] * vecn[nyz + f] + T[2] * vecn[2 * nyz + f]);
        h.Ts1[q] = (float)(T[0] * vecs1[f] + T[1] * vecs1[nyz + f] + T[2] * vecs1[2 * nyz + f]);
        h.Ts2[q] = (float)(T[0] * vecs2[f] + T[1] * vecs2[nyz + f] + T[2] * vecs2[2 * nyz + f]);
      }
  }
}

void FaultHost::resize(size_t nf) {
  for (auto* v : {&sx, &sy, &sz, &T0x, &T0y, &T0z, &dT0x, &dT0y, &dT0z, &str_peak, &Dc, &C0, &a, &b, &L, &Vw, &State,
                  &Tn, &Ts1, &Ts2, &init_t0})
    v->assign(nf, 0.0f);
  for (auto* v : {&united, &faultgrid, &rupy, &rupz}) v->assign(nf, 0);
}

}  // namespace dfd
