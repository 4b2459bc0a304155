// Configuration files in the .gro layout of the reference engine (host code).
// Reference: GromacsFileManager::readGroFile / writeGroFile
// (shortRange.inhomo/template/tools/simulation.hetero.cutoff/src/GromacsFileManager.cpp:7-124)
// and the callers MDSystem::initConfig / writeHostDataGro (src/MDSystem_interface.cu:39-215).
//
// Layout: a title line; the atom count; one line per atom with the residue
// index (5 columns), residue name (5), atom name (5), atom index (5), then the
// position (and optionally the velocity) as free-format numbers; the box edges.
// Names occupy fixed 8-byte slots (StringSize of the reference).  Numbers are
// parsed into binary32 and written from binary32, as the reference's
// ScalorType is float: a file read here gives exactly the reference's values,
// and a file written here is byte-identical to the reference's for the same
// binary32 state.
#include <cerrno>
#include <cstdio>
#include <cstring>
#include "../../include/mdforce.h"

void md_set_error(const char* fmt, ...);

namespace {

struct File {
  FILE* f = nullptr;
  explicit File(FILE* p) : f(p) {}
  ~File() { if (f) fclose(f); }
};

// a 5-column name field at line[off .. off+5), read like sscanf("%s") on it
bool name_field(const char* line, int off, char* out) {
  char tmp[8];
  size_t len = strlen(line);
  for (int j = 0; j < 5; ++j) tmp[j] = (size_t)(off + j) < len ? line[off + j] : '\0';
  tmp[5] = '\0';
  return sscanf(tmp, "%7s", out) == 1;
}

int bad_format(const char* path, const char* what) {
  md_set_error("wrong .gro format in %s: %s", path, what);
  return MD_ERR_IO;
}

}  // namespace

extern "C" int md_gro_count(const char* path, int* n_atoms) {
  if (!path || !n_atoms) return MD_ERR_BADARG;
  File fp(fopen(path, "r"));
  if (!fp.f) { md_set_error("cannot open %s: %s", path, strerror(errno)); return MD_ERR_IO; }
  char line[1024];
  int n = 0;
  if (!fgets(line, sizeof(line), fp.f) || !fgets(line, sizeof(line), fp.f) || sscanf(line, "%d", &n) != 1 || n < 0)
    return bad_format(path, "no atom count on line 2");
  *n_atoms = n;
  return MD_OK;
}

extern "C" int md_gro_read(const char* path, int n_atoms, int* resd_index, char* resd_name, char* atom_name,
                           int* atom_index, double* pos, double* vel, double box[3]) {
  if (!path || n_atoms < 0 || !pos || !box) return MD_ERR_BADARG;
  File fp(fopen(path, "r"));
  if (!fp.f) { md_set_error("cannot open %s: %s", path, strerror(errno)); return MD_ERR_IO; }
  char line[1024];
  int n = 0;
  if (!fgets(line, sizeof(line), fp.f) || !fgets(line, sizeof(line), fp.f) || sscanf(line, "%d", &n) != 1)
    return bad_format(path, "no atom count on line 2");
  if (n != n_atoms) {
    md_set_error("md_gro_read: %s holds %d atoms, the caller expects %d", path, n, n_atoms);
    return MD_ERR_BADARG;
  }
  for (int i = 0; i < n; ++i) {
    if (!fgets(line, sizeof(line), fp.f)) return bad_format(path, "fewer atom lines than the count");
    char s1[8], s2[8];
    if (!name_field(line, 5, s1) || !name_field(line, 10, s2)) return bad_format(path, "missing residue or atom name");
    int n1 = 0, n2 = 0;
    if (sscanf(line, "%5d", &n1) != 1) return bad_format(path, "missing residue index");
    if (strlen(line) < 15) return bad_format(path, "short atom line");
    float v[6];
    const int tag = sscanf(line + 15, "%5d%f%f%f%f%f%f", &n2, &v[0], &v[1], &v[2], &v[3], &v[4], &v[5]);
    if (tag != 7 && tag != 4) return bad_format(path, "an atom line needs a position and optionally a velocity");
    if (tag == 4) v[3] = v[4] = v[5] = 0.f;
    if (resd_index) resd_index[i] = n1;
    if (atom_index) atom_index[i] = n2;
    if (resd_name) { memset(resd_name + 8 * i, 0, 8); memcpy(resd_name + 8 * i, s1, strlen(s1)); }
    if (atom_name) { memset(atom_name + 8 * i, 0, 8); memcpy(atom_name + 8 * i, s2, strlen(s2)); }
    for (int d = 0; d < 3; ++d) {
      pos[3 * i + d] = (double)v[d];
      if (vel) vel[3 * i + d] = (double)v[3 + d];
    }
  }
  if (!fgets(line, sizeof(line), fp.f)) return bad_format(path, "no box line");
  float b[3];
  if (sscanf(line, "%f%f%f", &b[0], &b[1], &b[2]) != 3) return bad_format(path, "the box line needs three edges");
  for (int d = 0; d < 3; ++d) box[d] = (double)b[d];
  return MD_OK;
}

extern "C" int md_gro_write(const char* path, const char* title, int n_atoms, const int* resd_index,
                            const char* resd_name, const char* atom_name, const int* atom_index, const double* pos,
                            const double* vel, const double box[3]) {
  if (!path || n_atoms < 0 || !pos || !box) return MD_ERR_BADARG;
  File fp(fopen(path, "w"));
  if (!fp.f) { md_set_error("cannot open %s for writing: %s", path, strerror(errno)); return MD_ERR_IO; }
  if (title) fputs(title, fp.f);
  fprintf(fp.f, "\n%d\n", n_atoms);
  for (int i = 0; i < n_atoms; ++i) {
    char s1[9] = {0}, s2[9] = {0};
    if (resd_name) memcpy(s1, resd_name + 8 * i, 8);
    if (atom_name) memcpy(s2, atom_name + 8 * i, 8);
    const float x = (float)pos[3 * i], y = (float)pos[3 * i + 1], z = (float)pos[3 * i + 2];
    const float u = vel ? (float)vel[3 * i] : 0.f, v = vel ? (float)vel[3 * i + 1] : 0.f,
                w = vel ? (float)vel[3 * i + 2] : 0.f;
    fprintf(fp.f, "%5d%5s%5s%5d%8.3f%8.3f%8.3f%8.4f%8.4f%8.4f\n", resd_index ? resd_index[i] : i + 1, s1, s2,
            atom_index ? atom_index[i] : i + 1, x, y, z, u, v, w);
  }
  fprintf(fp.f, "%f %f %f\n", (float)box[0], (float)box[1], (float)box[2]);
  if (ferror(fp.f)) { md_set_error("write error on %s", path); return MD_ERR_IO; }
  return MD_OK;
}
