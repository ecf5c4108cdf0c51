// Output formats on the host side of the path: OVF vector fields and the
// ODT data table, as the reference's omf package writes them
// (src/go/mumax/omf/output.go:41-260, odt.go:103-131) for its autosaves and
// datatable.odt (src/go/sim/simoutput.go:161-272).
//
// A field is the engine's [3][X][Y][Z] float32 array (internal order, Z
// contiguous); the files are in user order: x, y, z = internal Z, Y, X, the
// vector components written x, y, z per cell, cells with x fastest (the
// internal C order read as Fortran order, output.go:199-201).  Binary data
// is "Binary 4": the control number 1234567.0 first, big-endian in OVF 1.0
// and little-endian in OVF 2.0 (output.go:208-260).  Numbers in text are
// written with nine significant digits (every float32 reads back exactly).
#include <stdio.h>
#include <string.h>

#include <string>
#include <vector>

#include "mmx_common.cuh"
#include "../../include/mmx.h"

namespace {

void put_be(FILE* f, float v) {
  unsigned char b[4];
  memcpy(b, &v, 4);
  unsigned char r[4] = {b[3], b[2], b[1], b[0]};
  fwrite(r, 1, 4, f);
}

void put_le(FILE* f, float v) {
  unsigned char b[4];
  memcpy(b, &v, 4);
  fwrite(b, 1, 4, f);
}

// "# Key: Value"
void hdr(FILE* f, const char* key, const std::string& val) { fprintf(f, "# %s: %s\n", key, val.c_str()); }
std::string num(double v) {
  char b[64];
  snprintf(b, sizeof b, "%.9g", v);
  return b;
}
std::string inum(long long v) { return std::to_string(v); }

}  // namespace

extern "C" int mmx_write_ovf(const char* path, const float* m, const int size[3], const double cellsize[3],
                             int ovf_version, int binary, const char* valueunit, double valuemultiplier,
                             double stage_time, double total_time) {
  if (!path || !m || !size || !cellsize || (ovf_version != 1 && ovf_version != 2)) {
    mmx_set_error("mmx_write_ovf: bad argument (ovf_version 1 or 2)");
    return MMX_ERR_ARG;
  }
  for (int d = 0; d < 3; d++)
    if (size[d] < 1) {
      mmx_set_error("mmx_write_ovf: size must be >= 1");
      return MMX_ERR_ARG;
    }
  FILE* f = fopen(path, "wb");
  if (!f) {
    mmx_set_error("mmx_write_ovf: cannot open the file");
    return MMX_ERR_ARG;
  }
  const int NX = size[2], NY = size[1], NZ = size[0];           // user x, y, z node counts
  const double cx = cellsize[2], cy = cellsize[1], cz = cellsize[0];
  const std::string unit = valueunit ? valueunit : "";
  // float32 products, as the Go code computes xmax = cellsize * float32(n)
  auto fmax = [](double c, int n) { return (double)((float)c * (float)n); };
  if (ovf_version == 1) {
    hdr(f, "OOMMF", "rectangular mesh v1.0");
    hdr(f, "Segment count", "1");
    hdr(f, "Begin", "Segment");
    hdr(f, "Begin", "Header");
    hdr(f, "Title", "mumax data");
    hdr(f, "meshtype", "rectangular");
    hdr(f, "meshunit", "m");
    hdr(f, "xbase", "0");
    hdr(f, "ybase", "0");
    hdr(f, "zbase", "0");
    hdr(f, "xstepsize", num((float)cx));
    hdr(f, "ystepsize", num((float)cy));
    hdr(f, "zstepsize", num((float)cz));
    hdr(f, "xmin", "0");
    hdr(f, "ymin", "0");
    hdr(f, "zmin", "0");
    hdr(f, "xmax", num(fmax(cx, NX)));
    hdr(f, "ymax", num(fmax(cy, NY)));
    hdr(f, "zmax", num(fmax(cz, NZ)));
    hdr(f, "xnodes", inum(NX));
    hdr(f, "ynodes", inum(NY));
    hdr(f, "znodes", inum(NZ));
    hdr(f, "ValueRangeMinMag", "1e-08");
    hdr(f, "ValueRangeMaxMag", "1");
    hdr(f, "valueunit", unit);
    hdr(f, "valuemultiplier", num(valuemultiplier));
    hdr(f, "End", "Header");
  } else {
    hdr(f, "OOMMF", "OVF 2.0");
    fprintf(f, "#\n");
    hdr(f, "Segment count", "1");
    fprintf(f, "#\n");
    hdr(f, "Begin", "Segment");
    hdr(f, "Begin", "Header");
    fprintf(f, "#\n");
    hdr(f, "title", "mumax data");
    hdr(f, "meshtype", "rectangular");
    hdr(f, "meshunit", "m");
    hdr(f, "xmin", "0");
    hdr(f, "ymin", "0");
    hdr(f, "zmin", "0");
    hdr(f, "xmax", num(fmax(cx, NX)));
    hdr(f, "ymax", num(fmax(cy, NY)));
    hdr(f, "zmax", num(fmax(cz, NZ)));
    hdr(f, "valuedim", "3");
    hdr(f, "valuelabels", "Val_x Val_y Val_z");
    hdr(f, "valueunits", unit + " " + unit + " " + unit);
    fprintf(f, "# desc: Stage simulation time:  %s  s\n", num(stage_time).c_str());
    fprintf(f, "# desc: Total simulation time:  %s  s\n", num(total_time).c_str());
    hdr(f, "xbase", num((float)cx / 2));
    hdr(f, "ybase", num((float)cy / 2));
    hdr(f, "zbase", num((float)cz / 2));
    hdr(f, "xnodes", inum(NX));
    hdr(f, "ynodes", inum(NY));
    hdr(f, "znodes", inum(NZ));
    hdr(f, "xstepsize", num((float)cx));
    hdr(f, "ystepsize", num((float)cy));
    hdr(f, "zstepsize", num((float)cz));
    fprintf(f, "#\n");
    hdr(f, "End", "Header");
    fprintf(f, "#\n");
  }
  const int64_t n = (int64_t)size[0] * size[1] * size[2];
  if (binary) {
    hdr(f, "Begin", "Data Binary 4");
    auto put = ovf_version == 1 ? put_be : put_le;
    put(f, 1234567.0f);
    for (int64_t g = 0; g < n; g++)
      for (int c = 2; c >= 0; c--) put(f, m[c * n + g]);
    hdr(f, "End", "Data Binary 4");
  } else {
    hdr(f, "Begin", "Data Text");
    for (int i = 0; i < size[0]; i++) {
      for (int j = 0; j < size[1]; j++) {
        for (int k = 0; k < size[2]; k++) {
          int64_t g = ((int64_t)i * size[1] + j) * size[2] + k;
          for (int c = 2; c >= 0; c--) fprintf(f, "%.9g ", m[c * n + g]);
          fprintf(f, "\t");
        }
        fprintf(f, "\n");
      }
      fprintf(f, "\n");
    }
    hdr(f, "End", "Data Text");
  }
  hdr(f, "End", "Segment");
  int bad = ferror(f);
  if (fclose(f) != 0 || bad) {
    mmx_set_error("mmx_write_ovf: write failed");
    return MMX_ERR_ARG;
  }
  return MMX_OK;
}

extern "C" int mmx_write_odt(const char* path, const float* rows, int nrows, const char* title) {
  if (!path || nrows < 0 || (nrows > 0 && !rows)) {
    mmx_set_error("mmx_write_odt: bad argument");
    return MMX_ERR_ARG;
  }
  FILE* f = fopen(path, "w");
  if (!f) {
    mmx_set_error("mmx_write_odt: cannot open the file");
    return MMX_ERR_ARG;
  }
  static const char* cols[7] = {"Time", "Mx/Ms", "My/Ms", "Mz/Ms", "max_dm/dt", "min_Mz/Ms", "max_Mz/Ms"};
  static const char* units[7] = {"s", "", "", "", "gammaMs", "", ""};
  fprintf(f, "# ODT 1.0\n");
  fprintf(f, "# Table Start\n");
  fprintf(f, "# Title:  %s\n", title ? title : "");
  fprintf(f, "# Units:");
  for (int c = 0; c < 7; c++) fprintf(f, "{%s} \t", units[c]);
  fprintf(f, "\n# Columns:");
  for (int c = 0; c < 7; c++) fprintf(f, "%s \t", cols[c]);
  fprintf(f, "\n");
  for (int r = 0; r < nrows; r++) {
    for (int c = 0; c < 7; c++) fprintf(f, "%-19.9g \t", rows[7 * (int64_t)r + c]);
    fprintf(f, "\n");
  }
  fprintf(f, "# Table End\n");
  int bad = ferror(f);
  if (fclose(f) != 0 || bad) {
    mmx_set_error("mmx_write_odt: write failed");
    return MMX_ERR_ARG;
  }
  return MMX_OK;
}
