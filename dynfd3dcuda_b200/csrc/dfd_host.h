// Host-side declarations shared by the C ABI implementation.
#pragma once
#include <cstddef>
#include <string>
#include <vector>

#include "../../include/dfd_b200.h"

namespace dfd {

struct FaultHost {
  std::vector<float> sx, sy, sz, T0x, T0y, T0z, dT0x, dT0y, dT0z, str_peak, Dc, C0, a, b, L, Vw, State, Tn, Ts1, Ts2,
      init_t0;
  std::vector<int> united, faultgrid, rupy, rupz;
  void resize(size_t nf);
};

void params_default(dfd_params* p);
void finalize_params(dfd_params* p);
int params_from_json(const char* text, dfd_params* p, std::string* err);
int check_params(const dfd_params* p, std::string* err);
void pml_profile(const dfd_params* p, int n, bool lo, bool hi, std::vector<float>& A, std::vector<float>& B,
                 std::vector<float>& D);
void cerjan_profile(const dfd_params* p, int npad, bool lo, bool hi, std::vector<float>& out);
void x_line(const dfd_params* p, std::vector<double>& xl);
void surface(const dfd_params* p, const float* fxyz, std::vector<double>& fx, std::vector<double>& fy,
             std::vector<double>& fz);
void fault_init(const dfd_params* p, const float* planes, const float* vecn, const float* vecs1, const float* vecs2,
                FaultHost& h);

// NetCDF classic (CDF-1/CDF-2) reader and writer -- dfd_netcdf.cpp
struct NcVar {
  std::string name;
  int type;  // 4 int, 5 float, 6 double
  std::vector<int> dims;
};
class NcWriter {
 public:
  bool open(const std::string& path);
  int dim(const std::string& name, long len);  // len 0 = unlimited (record) dimension
  int var(const std::string& name, int type, const std::vector<int>& dims);
  bool enddef();
  bool put_fixed(int varid, const void* data);                    // whole fixed-size variable
  bool put_record(int varid, long rec, const void* data);         // one record of a record variable
  bool sync();
  void close();
  ~NcWriter() { close(); }

 private:
  void* fp_ = nullptr;
  std::vector<std::pair<std::string, long>> dims_;
  std::vector<NcVar> vars_;
  std::vector<long long> begin_, vsize_;
  long long recsize_ = 0;
  long numrecs_ = 0;
  int recdim_ = -1;
  bool defined_ = false;
  void write_header();
};
// read a fixed (nz, ny) float variable of a classic file into out; false if missing
bool nc_read_plane(const std::string& path, const std::string& var, long nz, long ny, float* out, std::string* err);

}  // namespace dfd
