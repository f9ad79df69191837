// NetCDF classic (CDF-2, 64-bit offsets) writer and a reader for fixed-size variables,
// written from the public classic-format description.  Used for the reference's input
// files (Fault_geometry, Fault_init_stress) and its outputs (io_fault.cu:16-285,
// io_wave_xy.cu:9-188): record dimension "nt", big-endian data.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include "dfd_host.h"

namespace dfd {

static void be32(std::vector<unsigned char>& b, uint32_t v) {
  b.push_back(v >> 24); b.push_back(v >> 16); b.push_back(v >> 8); b.push_back(v);
}
static void be64(std::vector<unsigned char>& b, uint64_t v) { be32(b, (uint32_t)(v >> 32)); be32(b, (uint32_t)v); }
static void name(std::vector<unsigned char>& b, const std::string& s) {
  be32(b, (uint32_t)s.size());
  for (char c : s) b.push_back((unsigned char)c);
  while (b.size() % 4) b.push_back(0);
}

bool NcWriter::open(const std::string& path) {
  close();
  fp_ = fopen(path.c_str(), "w+b");
  dims_.clear(); vars_.clear(); begin_.clear(); vsize_.clear();
  numrecs_ = 0; recdim_ = -1; defined_ = false;
  return fp_ != nullptr;
}
int NcWriter::dim(const std::string& n, long len) {
  if (len == 0) recdim_ = (int)dims_.size();
  dims_.emplace_back(n, len);
  return (int)dims_.size() - 1;
}
int NcWriter::var(const std::string& n, int type, const std::vector<int>& dims) {
  vars_.push_back(NcVar{n, type, dims});
  return (int)vars_.size() - 1;
}
void NcWriter::write_header() {
  std::vector<unsigned char> b = {'C', 'D', 'F', 2};
  be32(b, (uint32_t)numrecs_);
  be32(b, 0x0A);
  be32(b, (uint32_t)dims_.size());
  for (auto& d : dims_) { name(b, d.first); be32(b, (uint32_t)d.second); }
  be32(b, 0); be32(b, 0);  // no global attributes
  be32(b, 0x0B);
  be32(b, (uint32_t)vars_.size());
  for (size_t v = 0; v < vars_.size(); v++) {
    name(b, vars_[v].name);
    be32(b, (uint32_t)vars_[v].dims.size());
    for (int d : vars_[v].dims) be32(b, (uint32_t)d);
    be32(b, 0); be32(b, 0);  // no attributes
    be32(b, (uint32_t)vars_[v].type);
    be32(b, (uint32_t)vsize_[v]);
    be64(b, (uint64_t)begin_[v]);
  }
  FILE* f = (FILE*)fp_;
  fseek(f, 0, SEEK_SET);
  fwrite(b.data(), 1, b.size(), f);
}
bool NcWriter::enddef() {
  if (!fp_) return false;
  // header size with placeholder offsets
  size_t hdr = 8 + 8;
  for (auto& d : dims_) hdr += 4 + (d.first.size() + 3) / 4 * 4 + 4;
  hdr += 8 + 8;
  for (auto& v : vars_) hdr += 4 + (v.name.size() + 3) / 4 * 4 + 4 + 4 * v.dims.size() + 8 + 4 + 4 + 8;
  begin_.assign(vars_.size(), 0);
  vsize_.assign(vars_.size(), 0);
  long long off = (long long)hdr;
  for (size_t v = 0; v < vars_.size(); v++) {  // fixed variables first
    bool rec = !vars_[v].dims.empty() && vars_[v].dims[0] == recdim_;
    long long n = 4;
    for (size_t d = rec ? 1 : 0; d < vars_[v].dims.size(); d++) n *= dims_[vars_[v].dims[d]].second;
    vsize_[v] = (n + 3) / 4 * 4;
    if (!rec) { begin_[v] = off; off += vsize_[v]; }
  }
  recsize_ = 0;
  for (size_t v = 0; v < vars_.size(); v++) {
    bool rec = !vars_[v].dims.empty() && vars_[v].dims[0] == recdim_;
    if (rec) { begin_[v] = off + recsize_; recsize_ += vsize_[v]; }
  }
  defined_ = true;
  write_header();
  return true;
}
static void write_be(FILE* f, long long off, const void* data, long long nbytes) {
  const uint32_t* s = (const uint32_t*)data;
  std::vector<uint32_t> tmp((size_t)(nbytes / 4));
  for (size_t i = 0; i < tmp.size(); i++) tmp[i] = __builtin_bswap32(s[i]);
  fseek(f, (long)off, SEEK_SET);
  fwrite(tmp.data(), 4, tmp.size(), f);
}
bool NcWriter::put_fixed(int v, const void* data) {
  if (!defined_) return false;
  write_be((FILE*)fp_, begin_[v], data, vsize_[v]);
  return true;
}
bool NcWriter::put_record(int v, long rec, const void* data) {
  if (!defined_) return false;
  write_be((FILE*)fp_, begin_[v] + rec * recsize_, data, vsize_[v]);
  if (rec + 1 > numrecs_) numrecs_ = rec + 1;
  return true;
}
bool NcWriter::sync() {
  if (!fp_) return false;
  write_header();
  fflush((FILE*)fp_);
  return true;
}
void NcWriter::close() {
  if (fp_) {
    if (defined_) write_header();
    fclose((FILE*)fp_);
    fp_ = nullptr;
  }
}

// ---------------------------------------------------------------- reader ----
static uint32_t rd32(FILE* f) {
  unsigned char b[4] = {0, 0, 0, 0};
  if (fread(b, 1, 4, f) != 4) return 0;
  return ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
}
static std::string rdname(FILE* f) {
  uint32_t n = rd32(f);
  std::string s(n, '\0');
  if (n && fread(&s[0], 1, n, f) != n) return "";
  fseek(f, (long)((4 - n % 4) % 4), SEEK_CUR);
  return s;
}
static int tsize(int t) { return t == 1 || t == 2 ? 1 : t == 3 ? 2 : t == 6 ? 8 : 4; }
static void skip_atts(FILE* f) {
  uint32_t tag = rd32(f), n = rd32(f);
  if (!tag) return;
  for (uint32_t a = 0; a < n; a++) {
    rdname(f);
    int t = (int)rd32(f);
    uint64_t bytes = (uint64_t)rd32(f) * tsize(t);
    fseek(f, (long)(bytes + (4 - bytes % 4) % 4), SEEK_CUR);
  }
}

bool nc_read_plane(const std::string& path, const std::string& var, long nz, long ny, float* out, std::string* err) {
  FILE* f = fopen(path.c_str(), "rb");
  if (!f) { if (err) *err = "cannot open " + path; return false; }
  unsigned char mg[4];
  if (fread(mg, 1, 4, f) != 4 || mg[0] != 'C' || mg[1] != 'D' || mg[2] != 'F' || (mg[3] != 1 && mg[3] != 2)) {
    fclose(f);
    if (err) *err = path + " is not a NetCDF classic file";
    return false;
  }
  bool v2 = mg[3] == 2;
  rd32(f);
  std::vector<long> dimlen;
  uint32_t tag = rd32(f), n = rd32(f);
  if (tag) for (uint32_t d = 0; d < n; d++) { rdname(f); dimlen.push_back(rd32(f)); }
  skip_atts(f);
  tag = rd32(f); n = rd32(f);
  bool found = false;
  for (uint32_t v = 0; v < n && tag; v++) {
    std::string nm = rdname(f);
    uint32_t nd = rd32(f);
    long long total = 1;
    for (uint32_t d = 0; d < nd; d++) total *= dimlen[rd32(f)];
    skip_atts(f);
    int t = (int)rd32(f);
    rd32(f);
    uint64_t begin = v2 ? ((uint64_t)rd32(f) << 32 | rd32(f)) : rd32(f);
    if (nm != var) continue;
    found = true;
    if (total != nz * ny || (t != 5 && t != 6)) {
      fclose(f);
      if (err) *err = var + " in " + path + " has the wrong size or type";
      return false;
    }
    long pos = ftell(f);
    fseek(f, (long)begin, SEEK_SET);
    std::vector<unsigned char> buf((size_t)total * tsize(t));
    if (fread(buf.data(), 1, buf.size(), f) != buf.size()) { fclose(f); if (err) *err = "short read"; return false; }
    for (long long i = 0; i < total; i++) {
      if (t == 5) {
        uint32_t u;
        memcpy(&u, &buf[4 * i], 4);
        u = __builtin_bswap32(u);
        memcpy(&out[i], &u, 4);
      } else {
        uint64_t u;
        memcpy(&u, &buf[8 * i], 8);
        u = __builtin_bswap64(u);
        double dv;
        memcpy(&dv, &u, 8);
        out[i] = (float)dv;
      }
    }
    fseek(f, pos, SEEK_SET);
    break;
  }
  fclose(f);
  if (!found && err) *err = "variable " + var + " not found in " + path;
  return found;
}

}  // namespace dfd
