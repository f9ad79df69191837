/* NetCDF-classic shim -- test infrastructure only.
 * Declares the entry points the reference's sources call (nc_open ..
 * nc_put_var_int).  The reading side is implemented from the public
 * classic (CDF-1 / CDF-2) format description; the writing side is not needed by
 * the harness and reports an error if reached. */
#ifndef DFD_REFSHIM_NETCDF_H
#define DFD_REFSHIM_NETCDF_H
#include <stddef.h>
#ifdef __cplusplus
extern "C" {
#endif
typedef int nc_type;
#define NC_NOERR 0
#define NC_NOWRITE 0
#define NC_CLOBBER 0
#define NC_UNLIMITED 0L
#define NC_BYTE 1
#define NC_CHAR 2
#define NC_SHORT 3
#define NC_INT 4
#define NC_FLOAT 5
#define NC_DOUBLE 6
int nc_open(const char *path, int mode, int *ncid);
int nc_create(const char *path, int mode, int *ncid);
int nc_close(int ncid);
int nc_sync(int ncid);
int nc_enddef(int ncid);
const char *nc_strerror(int err);
int nc_inq_varid(int ncid, const char *name, int *varid);
int nc_def_dim(int ncid, const char *name, size_t len, int *dimid);
int nc_def_var(int ncid, const char *name, nc_type t, int nd, const int *dimids, int *varid);
int nc_get_vara_float(int ncid, int varid, const size_t *start, const size_t *count, float *out);
int nc_get_vara_double(int ncid, int varid, const size_t *start, const size_t *count, double *out);
int nc_put_vara_float(int ncid, int varid, const size_t *start, const size_t *count, const float *in);
int nc_put_vara_double(int ncid, int varid, const size_t *start, const size_t *count, const double *in);
int nc_put_vara_int(int ncid, int varid, const size_t *start, const size_t *count, const int *in);
int nc_put_var_float(int ncid, int varid, const float *in);
int nc_put_var_double(int ncid, int varid, const double *in);
int nc_put_var_int(int ncid, int varid, const int *in);
#ifdef __cplusplus
}
#endif
#endif
