// host_restart.cpp -- restart files in the layout of the reference's IOSCALAR
// (src/io.f:114-200), serial case: Fortran unformatted sequential records,
// each framed by a 4-byte little-endian length before and after (the gfortran
// record marker):
//   NX, NY, NZ, 1            four int32
//   A(1:NX,1:NY,k)           NX*NY float64, one record per k = 1..NZ
//   nstep                    int32
//   TIME                     float64
//   DTM1, grav               two float64
// Host-only: the device entry points (eddy_save_field / eddy_load_field) copy
// through a host buffer around these.
//
// Also the inflow-plane files of the hybrid inlet (read_hybrid,
// src/hybrid.f:162-200), the same record framing:
//   icycle                                   int32
//   TIME, DTM1, grav, rho, Re, Pr            six float64
//   dir, (unused), index                     three int32
//   zcg, zwg                                 two float64
//   NX, (unused), NY                         three int32
//   xc(1:NX), xu(1:NX)                       2 NX float64
//   yc(1:NY), yv(1:NY)                       2 NY float64
//   planeU, planeV, planeW, planeP, planeD   NX*NY float64 each
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/eddy_b200.h"

namespace {

bool put_record(FILE *f, const void *data, uint32_t bytes) {
  return fwrite(&bytes, 4, 1, f) == 1 && (bytes == 0 || fwrite(data, 1, bytes, f) == bytes) &&
         fwrite(&bytes, 4, 1, f) == 1;
}

// reads one record of exactly `bytes` payload bytes
bool get_record(FILE *f, void *data, uint32_t bytes) {
  uint32_t a = 0, b = 0;
  if (fread(&a, 4, 1, f) != 1 || a != bytes) return false;
  if (bytes && fread(data, 1, bytes, f) != bytes) return false;
  return fread(&b, 4, 1, f) == 1 && b == bytes;
}

}  // namespace

extern "C" int eddy_ioscalar_write(const char *path, int nx, int ny, int nz, const double *a, int nstep,
                                   double time, double dtm1, double grav) {
  if (!path || !a || nx < 1 || ny < 1 || nz < 1) return EDDY_EINVAL;
  const uint64_t plane = (uint64_t)nx * ny * sizeof(double);
  if (plane > 0x7fffffffu) return EDDY_EINVAL;  // one record per plane must fit a 4-byte marker
  FILE *f = fopen(path, "wb");
  if (!f) return EDDY_EINVAL;
  const int32_t hdr[4] = {nx, ny, nz, 1};
  bool ok = put_record(f, hdr, sizeof hdr);
  for (int k = 0; ok && k < nz; k++) ok = put_record(f, a + (size_t)k * nx * ny, (uint32_t)plane);
  const int32_t ns = nstep;
  const double t2[2] = {dtm1, grav};
  ok = ok && put_record(f, &ns, 4) && put_record(f, &time, 8) && put_record(f, t2, 16);
  ok = (fclose(f) == 0) && ok;
  return ok ? EDDY_OK : EDDY_EINVAL;
}

extern "C" int eddy_ioscalar_read(const char *path, int nx, int ny, int nz, double *a, int *nstep, double *time,
                                  double *dtm1, double *grav) {
  if (!path || !a || nx < 1 || ny < 1 || nz < 1) return EDDY_EINVAL;
  FILE *f = fopen(path, "rb");
  if (!f) return EDDY_EINVAL;
  int32_t hdr[4] = {0, 0, 0, 0};
  // the reference reads the header and does not check it; a file of another
  // grid is refused here
  bool ok = get_record(f, hdr, sizeof hdr) && hdr[0] == nx && hdr[1] == ny && hdr[2] == nz;
  const uint32_t plane = (uint32_t)((uint64_t)nx * ny * sizeof(double));
  for (int k = 0; ok && k < nz; k++) ok = get_record(f, a + (size_t)k * nx * ny, plane);
  int32_t ns = 0;
  double t = 0., t2[2] = {0., 0.};
  ok = ok && get_record(f, &ns, 4) && get_record(f, &t, 8) && get_record(f, t2, 16);
  fclose(f);
  if (!ok) return EDDY_EINVAL;
  if (nstep) *nstep = ns;
  if (time) *time = t;
  if (dtm1) *dtm1 = t2[0];
  if (grav) *grav = t2[1];
  return EDDY_OK;
}

extern "C" int eddy_read_hybrid_plane(const char *path, int nx, int ny, double *u, double *v, double *w, double *p,
                                      double *d, int *icycle, double *time) {
  if (!path || nx < 1 || ny < 1) return EDDY_EINVAL;
  const uint64_t n2 = (uint64_t)nx * ny;
  if (n2 * sizeof(double) > 0x7fffffffu) return EDDY_EINVAL;
  FILE *f = fopen(path, "rb");
  if (!f) return EDDY_EINVAL;
  int32_t ic = 0, i3[3] = {0, 0, 0}, dims[3] = {0, 0, 0};
  double t6[6], z2[2];
  std::vector<double> axes(2 * (size_t)(nx > ny ? nx : ny)), plane(n2);
  bool ok = get_record(f, &ic, 4) && get_record(f, t6, sizeof t6) && get_record(f, i3, sizeof i3) &&
            get_record(f, z2, sizeof z2) && get_record(f, dims, sizeof dims);
  // a plane of another grid is refused (the reference reads it unchecked)
  ok = ok && dims[0] == nx && dims[2] == ny;
  ok = ok && get_record(f, axes.data(), (uint32_t)(2 * nx * sizeof(double))) &&
       get_record(f, axes.data(), (uint32_t)(2 * ny * sizeof(double)));
  double *out[5] = {u, v, w, p, d};
  for (int q = 0; ok && q < 5; q++) {
    ok = get_record(f, plane.data(), (uint32_t)(n2 * sizeof(double)));
    if (ok && out[q]) memcpy(out[q], plane.data(), n2 * sizeof(double));
  }
  fclose(f);
  if (!ok) return EDDY_EINVAL;
  if (icycle) *icycle = ic;
  if (time) *time = t6[0];
  return EDDY_OK;
}
