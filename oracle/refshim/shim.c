/* Implementation of the single-rank MPI shim and the read-only NetCDF-classic
 * shim declared in mpi.h / netcdf.h -- test infrastructure only. */
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>
#include "mpi.h"
#include "netcdf.h"

/* ---------------------------------------------------------------- MPI ---- */
int MPI_Init(int *argc, char ***argv) { (void)argc; (void)argv; return 0; }
int MPI_Finalize(void) { return 0; }
int MPI_Comm_rank(MPI_Comm c, int *r) { (void)c; *r = 0; return 0; }
int MPI_Comm_size(MPI_Comm c, int *s) { (void)c; *s = 1; return 0; }
int MPI_Get_processor_name(char *name, int *len) { strcpy(name, "shim"); *len = 4; return 0; }
int MPI_Cart_create(MPI_Comm c, int nd, const int *dims, const int *periods, int reorder, MPI_Comm *out) {
  (void)c; (void)nd; (void)dims; (void)periods; (void)reorder; *out = 0; return 0;
}
int MPI_Cart_coords(MPI_Comm c, int rank, int nd, int *coords) {
  (void)c; (void)rank; for (int i = 0; i < nd; i++) coords[i] = 0; return 0;
}
int MPI_Cart_shift(MPI_Comm c, int dir, int disp, int *src, int *dst) {
  (void)c; (void)dir; (void)disp; *src = MPI_PROC_NULL; *dst = MPI_PROC_NULL; return 0;
}
int MPI_Barrier(MPI_Comm c) { (void)c; return 0; }
int MPI_Abort(MPI_Comm c, int code) { (void)c; fprintf(stderr, "MPI_Abort(%d)\n", code); exit(code); }
int MPI_Reduce(const void *in, void *out, int n, MPI_Datatype t, MPI_Op op, int root, MPI_Comm c) {
  (void)op; (void)root; (void)c;
  size_t sz = t == MPI_DOUBLE ? 8 : 4;
  memcpy(out, in, sz * (size_t)n);
  return 0;
}
int MPI_Sendrecv(const void *sb, int sn, MPI_Datatype st, int dst, int stag, void *rb, int rn, MPI_Datatype rt,
                 int src, int rtag, MPI_Comm c, MPI_Status *status) {
  (void)sb; (void)sn; (void)st; (void)dst; (void)stag; (void)rb; (void)rn; (void)rt; (void)src; (void)rtag;
  (void)c; (void)status;
  fprintf(stderr, "MPI_Sendrecv reached in a single-rank shim\n");
  return 1;
}

/* ------------------------------------------------------ NetCDF classic ---- */
#define MAXF 16
#define MAXV 64
#define MAXD 16
typedef struct {
  char name[128];
  int nd, dimids[8];
  int type;
  uint64_t begin;
} ncvar;
typedef struct {
  FILE *fp;
  int ndims;
  uint64_t dimlen[MAXD];
  int nvars;
  ncvar vars[MAXV];
} ncfile;
static ncfile *files[MAXF];

static uint32_t rd32(FILE *f) {
  unsigned char b[4];
  if (fread(b, 1, 4, f) != 4) return 0;
  return ((uint32_t)b[0] << 24) | ((uint32_t)b[1] << 16) | ((uint32_t)b[2] << 8) | b[3];
}
static uint64_t rd64(FILE *f) {
  uint64_t hi = rd32(f);
  return (hi << 32) | rd32(f);
}
static void rdname(FILE *f, char *out, size_t cap) {
  uint32_t n = rd32(f);
  uint32_t pad = (4 - n % 4) % 4;
  size_t keep = n < cap - 1 ? n : cap - 1;
  if (fread(out, 1, keep, f) != keep) keep = 0;
  out[keep] = 0;
  fseek(f, (long)(n - keep + pad), SEEK_CUR);
}
static int tsize(int t) { return t == 1 || t == 2 ? 1 : t == 3 ? 2 : t == 6 ? 8 : 4; }
static void skip_atts(FILE *f) {
  uint32_t tag = rd32(f), n = rd32(f);
  if (tag == 0) return;
  for (uint32_t a = 0; a < n; a++) {
    char nm[256];
    rdname(f, nm, sizeof nm);
    int t = (int)rd32(f);
    uint32_t cnt = rd32(f);
    uint64_t bytes = (uint64_t)cnt * tsize(t);
    fseek(f, (long)(bytes + (4 - bytes % 4) % 4), SEEK_CUR);
  }
}
int nc_open(const char *path, int mode, int *ncid) {
  (void)mode;
  FILE *f = fopen(path, "rb");
  if (!f) return -31;
  char mg[4];
  if (fread(mg, 1, 4, f) != 4 || mg[0] != 'C' || mg[1] != 'D' || mg[2] != 'F' || (mg[3] != 1 && mg[3] != 2)) {
    fclose(f);
    return -51;
  }
  int v2 = mg[3] == 2;
  ncfile *nc = (ncfile *)calloc(1, sizeof(ncfile));
  nc->fp = f;
  rd32(f); /* numrecs */
  uint32_t tag = rd32(f), n = rd32(f);
  if (tag != 0) {
    nc->ndims = (int)n;
    for (uint32_t d = 0; d < n && d < MAXD; d++) {
      char nm[256];
      rdname(f, nm, sizeof nm);
      nc->dimlen[d] = rd32(f);
    }
  }
  skip_atts(f);
  tag = rd32(f);
  n = rd32(f);
  if (tag != 0) {
    nc->nvars = (int)n;
    for (uint32_t v = 0; v < n && v < MAXV; v++) {
      ncvar *var = &nc->vars[v];
      rdname(f, var->name, sizeof var->name);
      var->nd = (int)rd32(f);
      for (int d = 0; d < var->nd; d++) var->dimids[d] = (int)rd32(f);
      skip_atts(f);
      var->type = (int)rd32(f);
      rd32(f); /* vsize */
      var->begin = v2 ? rd64(f) : rd32(f);
    }
  }
  for (int i = 0; i < MAXF; i++)
    if (!files[i]) { files[i] = nc; *ncid = i; return NC_NOERR; }
  fclose(f);
  free(nc);
  return -1;
}
int nc_close(int ncid) {
  if (ncid < 0 || ncid >= MAXF || !files[ncid]) return -33;
  fclose(files[ncid]->fp);
  free(files[ncid]);
  files[ncid] = NULL;
  return NC_NOERR;
}
int nc_inq_varid(int ncid, const char *name, int *varid) {
  if (ncid < 0 || ncid >= MAXF || !files[ncid]) return -33;
  for (int v = 0; v < files[ncid]->nvars; v++)
    if (!strcmp(files[ncid]->vars[v].name, name)) { *varid = v; return NC_NOERR; }
  return -49;
}
/* hyperslab read of a fixed-size variable, converted to double */
static int get_vara(int ncid, int varid, const size_t *start, const size_t *count, double *out) {
  if (ncid < 0 || ncid >= MAXF || !files[ncid]) return -33;
  ncfile *nc = files[ncid];
  if (varid < 0 || varid >= nc->nvars) return -49;
  ncvar *v = &nc->vars[varid];
  int ts = tsize(v->type);
  uint64_t shape[8], total = 1;
  for (int d = 0; d < v->nd; d++) {
    shape[d] = nc->dimlen[v->dimids[d]];
    if (start[d] + count[d] > shape[d]) return -40;
    total *= count[d];
  }
  uint64_t idx[8] = {0};
  unsigned char buf[8];
  for (uint64_t n = 0; n < total; n++) {
    uint64_t off = 0;
    for (int d = 0; d < v->nd; d++) off = off * shape[d] + start[d] + idx[d];
    fseek(nc->fp, (long)(v->begin + off * ts), SEEK_SET);
    if (fread(buf, 1, ts, nc->fp) != (size_t)ts) return -52;
    double val = 0;
    if (v->type == NC_FLOAT) {
      uint32_t u = ((uint32_t)buf[0] << 24) | ((uint32_t)buf[1] << 16) | ((uint32_t)buf[2] << 8) | buf[3];
      float fv;
      memcpy(&fv, &u, 4);
      val = fv;
    } else if (v->type == NC_DOUBLE) {
      uint64_t u = 0;
      for (int b = 0; b < 8; b++) u = (u << 8) | buf[b];
      memcpy(&val, &u, 8);
    } else if (v->type == NC_INT) {
      int32_t iv = (int32_t)(((uint32_t)buf[0] << 24) | ((uint32_t)buf[1] << 16) | ((uint32_t)buf[2] << 8) | buf[3]);
      val = iv;
    } else {
      return -45;
    }
    out[n] = val;
    for (int d = v->nd - 1; d >= 0; d--) {
      if (++idx[d] < count[d]) break;
      idx[d] = 0;
    }
  }
  return NC_NOERR;
}
static uint64_t prod(int ncid, int varid, const size_t *count) {
  uint64_t t = 1;
  for (int d = 0; d < files[ncid]->vars[varid].nd; d++) t *= count[d];
  return t;
}
int nc_get_vara_double(int ncid, int varid, const size_t *start, const size_t *count, double *out) {
  return get_vara(ncid, varid, start, count, out);
}
int nc_get_vara_float(int ncid, int varid, const size_t *start, const size_t *count, float *out) {
  if (ncid < 0 || ncid >= MAXF || !files[ncid] || varid < 0 || varid >= files[ncid]->nvars) return -49;
  uint64_t n = prod(ncid, varid, count);
  double *tmp = (double *)malloc(sizeof(double) * (n ? n : 1));
  int e = get_vara(ncid, varid, start, count, tmp);
  for (uint64_t i = 0; e == NC_NOERR && i < n; i++) out[i] = (float)tmp[i];
  free(tmp);
  return e;
}
const char *nc_strerror(int err) {
  static char msg[64];
  snprintf(msg, sizeof msg, "netcdf shim error %d", err);
  return msg;
}
/* writing is not part of the harness */
int nc_create(const char *p, int m, int *id) { (void)p; (void)m; (void)id; return -128; }
int nc_sync(int id) { (void)id; return NC_NOERR; }
int nc_enddef(int id) { (void)id; return -128; }
int nc_def_dim(int id, const char *n, size_t l, int *d) { (void)id; (void)n; (void)l; (void)d; return -128; }
int nc_def_var(int id, const char *n, nc_type t, int nd, const int *di, int *v) {
  (void)id; (void)n; (void)t; (void)nd; (void)di; (void)v; return -128;
}
int nc_put_vara_float(int a, int b, const size_t *s, const size_t *c, const float *i) {
  (void)a; (void)b; (void)s; (void)c; (void)i; return -128;
}
int nc_put_vara_double(int a, int b, const size_t *s, const size_t *c, const double *i) {
  (void)a; (void)b; (void)s; (void)c; (void)i; return -128;
}
int nc_put_vara_int(int a, int b, const size_t *s, const size_t *c, const int *i) {
  (void)a; (void)b; (void)s; (void)c; (void)i; return -128;
}
int nc_put_var_float(int a, int b, const float *i) { (void)a; (void)b; (void)i; return -128; }
int nc_put_var_double(int a, int b, const double *i) { (void)a; (void)b; (void)i; return -128; }
int nc_put_var_int(int a, int b, const int *i) { (void)a; (void)b; (void)i; return -128; }
