// io.cu -- checkpoint files of the primitive grids (grid::dump and
// grid::load, grid.cpp:367-381 and 482-499) as host-side format code; the
// handle-level dump / load / restart calls in runtime.cu use it.
//
// The reference writes a grid with PETSc's HDF5 viewer: VecView of the
// DMDA global vector, i.e. the interior zones in natural order with the
// variables interleaved ([k][j][i][var], var fastest).  HDF5 is not linked
// into this library, so the same vector, in the same order, is written in
// PETSc's binary Vec format (PetscViewerBinary + VecView / VecLoad, with
// 32-bit PetscInt):
//   int32  VEC_FILE_CLASSID = 1211214   big-endian
//   int32  number of entries            big-endian
//   double entries[n]                   big-endian IEEE 754
// PETSc's VecLoad (PetscViewerBinaryOpen) and PetscBinaryIO read it.
#include <cstdint>
#include <cstdio>
#include <cstring>
#include <vector>

#include "../../include/grim_b200.h"

namespace grim {
void set_error_message(const char* msg);
}

namespace {
const int32_t kVecClassId = 1211214;

bool little_endian() {
  const uint16_t one = 1;
  unsigned char b;
  std::memcpy(&b, &one, 1);
  return b == 1;
}
void swap8(unsigned char* p) {
  for (int a = 0, b = 7; a < b; a++, b--) {
    const unsigned char t = p[a];
    p[a] = p[b];
    p[b] = t;
  }
}
void put_be32(unsigned char* p, int32_t v) {
  const uint32_t u = (uint32_t)v;
  p[0] = (unsigned char)(u >> 24); p[1] = (unsigned char)(u >> 16);
  p[2] = (unsigned char)(u >> 8); p[3] = (unsigned char)u;
}
int32_t get_be32(const unsigned char* p) {
  return (int32_t)(((uint32_t)p[0] << 24) | ((uint32_t)p[1] << 16) | ((uint32_t)p[2] << 8) | (uint32_t)p[3]);
}

// zone counts of a configuration (ghosts on the active dimensions only)
struct Shape {
  int N1, N2, N3, g1, g2, g3, N1T, N2T, N3T, dof;
};
bool shape_of(const grim_config* c, Shape& s) {
  if (!c || c->dim < 1 || c->dim > 3 || c->N1 < 1 || c->numGhost < 0) return false;
  s.N1 = c->N1;
  s.N2 = c->dim >= 2 ? c->N2 : 1;
  s.N3 = c->dim >= 3 ? c->N3 : 1;
  if (s.N2 < 1 || s.N3 < 1) return false;
  s.g1 = c->numGhost;
  s.g2 = c->dim >= 2 ? c->numGhost : 0;
  s.g3 = c->dim >= 3 ? c->numGhost : 0;
  s.N1T = s.N1 + 2 * s.g1;
  s.N2T = s.N2 + 2 * s.g2;
  s.N3T = s.N3 + 2 * s.g3;
  s.dof = 8 + (c->conduction ? 1 : 0) + (c->viscosity ? 1 : 0);
  return true;
}
}  // namespace

extern "C" {

int grim_petsc_vec_write(const char* fileName, const double* v, long long n) {
  if (!fileName || (!v && n > 0) || n < 0 || n > 0x7fffffffLL) {
    grim::set_error_message("grim_petsc_vec_write: bad argument (n must fit a 32-bit PetscInt)");
    return GRIM_EINVAL;
  }
  FILE* f = std::fopen(fileName, "wb");
  if (!f) {
    grim::set_error_message("grim_petsc_vec_write: cannot open the file for writing");
    return GRIM_EINVAL;
  }
  unsigned char head[8];
  put_be32(head, kVecClassId);
  put_be32(head + 4, (int32_t)n);
  bool ok = std::fwrite(head, 1, 8, f) == 8;
  const bool swap = little_endian();
  std::vector<unsigned char> buf;
  const long long chunk = 1 << 16;
  for (long long a = 0; ok && a < n; a += chunk) {
    const long long m = (n - a < chunk) ? n - a : chunk;
    buf.resize((size_t)m * 8);
    std::memcpy(buf.data(), v + a, (size_t)m * 8);
    if (swap)
      for (long long q = 0; q < m; q++) swap8(buf.data() + q * 8);
    ok = std::fwrite(buf.data(), 1, buf.size(), f) == buf.size();
  }
  ok = (std::fclose(f) == 0) && ok;
  if (!ok) {
    grim::set_error_message("grim_petsc_vec_write: write failed");
    return GRIM_EINVAL;
  }
  return GRIM_OK;
}

int grim_petsc_vec_read(const char* fileName, double* v, long long n) {
  if (!fileName || (!v && n > 0) || n < 0) {
    grim::set_error_message("grim_petsc_vec_read: bad argument");
    return GRIM_EINVAL;
  }
  FILE* f = std::fopen(fileName, "rb");
  if (!f) {
    grim::set_error_message("grim_petsc_vec_read: cannot open the file");
    return GRIM_EINVAL;
  }
  unsigned char head[8];
  const size_t got = std::fread(head, 1, 8, f);
  // HDF5 files start with the signature \x89 H D F \r \n \x1a \n (at offset 0
  // when no user block precedes it): the reference's own restart files
  // (PETSc's HDF5 viewer, grid.cpp:367-381) are of that kind
  static const unsigned char kHdf5Sig[8] = {0x89, 'H', 'D', 'F', '\r', '\n', 0x1a, '\n'};
  if (got == 8 && std::memcmp(head, kHdf5Sig, 8) == 0) {
    std::fclose(f);
    grim::set_error_message(
        "grim_petsc_vec_read: this is an HDF5 file (such as the reference's restart file written with PETSc's HDF5 "
        "viewer); HDF5 restart files are not supported: this library reads PETSc binary Vec files only");
    return GRIM_ENOTSUP;
  }
  if (got != 8 || get_be32(head) != kVecClassId) {
    std::fclose(f);
    grim::set_error_message("grim_petsc_vec_read: not a PETSc binary Vec (class id 1211214)");
    return GRIM_EINVAL;
  }
  if ((long long)get_be32(head + 4) != n) {
    std::fclose(f);
    char msg[160];
    std::snprintf(msg, sizeof(msg), "grim_petsc_vec_read: the file holds %d entries, the grid needs %lld",
                  (int)get_be32(head + 4), n);
    grim::set_error_message(msg);
    return GRIM_EINVAL;
  }
  const bool swap = little_endian();
  std::vector<unsigned char> buf;
  const long long chunk = 1 << 16;
  bool ok = true;
  for (long long a = 0; ok && a < n; a += chunk) {
    const long long m = (n - a < chunk) ? n - a : chunk;
    buf.resize((size_t)m * 8);
    ok = std::fread(buf.data(), 1, buf.size(), f) == buf.size();
    if (!ok) break;
    if (swap)
      for (long long q = 0; q < m; q++) swap8(buf.data() + q * 8);
    std::memcpy(v + a, buf.data(), (size_t)m * 8);
  }
  std::fclose(f);
  if (!ok) {
    grim::set_error_message("grim_petsc_vec_read: the file is shorter than its header says");
    return GRIM_EINVAL;
  }
  return GRIM_OK;
}

int grim_natural_from_prims(const grim_config* cfg, const double* prims, double* natural) {
  Shape s;
  if (!shape_of(cfg, s) || !prims || !natural) {
    grim::set_error_message("grim_natural_from_prims: bad argument");
    return GRIM_EINVAL;
  }
  const long long Z = (long long)s.N1T * s.N2T * s.N3T;
  long long o = 0;
  for (int k = 0; k < s.N3; k++)
    for (int j = 0; j < s.N2; j++)
      for (int i = 0; i < s.N1; i++) {
        const long long z = (long long)(i + s.g1) + (long long)s.N1T * ((j + s.g2) + (long long)s.N2T * (k + s.g3));
        for (int v = 0; v < s.dof; v++) natural[o++] = prims[(long long)v * Z + z];
      }
  return GRIM_OK;
}

int grim_prims_from_natural(const grim_config* cfg, const double* natural, double* prims) {
  Shape s;
  if (!shape_of(cfg, s) || !prims || !natural) {
    grim::set_error_message("grim_prims_from_natural: bad argument");
    return GRIM_EINVAL;
  }
  const long long Z = (long long)s.N1T * s.N2T * s.N3T;
  long long o = 0;
  for (int k = 0; k < s.N3; k++)
    for (int j = 0; j < s.N2; j++)
      for (int i = 0; i < s.N1; i++) {
        const long long z = (long long)(i + s.g1) + (long long)s.N1T * ((j + s.g2) + (long long)s.N2T * (k + s.g3));
        for (int v = 0; v < s.dof; v++) prims[(long long)v * Z + z] = natural[o++];
      }
  return GRIM_OK;
}

}  // extern "C"
