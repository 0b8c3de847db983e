// Mesh I/O of the host driver: the gmsh 2.2 reader (host_mesh_read_msh,
// euler.c:556-833), the MFEM mesh writer (host_mesh_write_mfem,
// euler.c:1771-1857) and a gmsh 2.2 writer for meshes generated here.
//
// Reader semantics follow the reference: ASCII gmsh 2.x; $Nodes give the
// vertex coordinates (the first dim of them); $Elements keep the elements of
// type 2 (triangle, dim 2) or 4 (tetrahedron, dim 3) and skip every other
// type and the tags; $Periodic is skipped (euler.c:658-686 turns it off:
// periodicity comes from matching the boundary of the vertices' bounding box,
// euler.c:3013-3050, which is the box returned here).  Additionally, an
// element whose vertex order is negatively oriented gets its vertices 1 and 2
// swapped, since the geometric factors assume positive orientation.
#include <cerrno>
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <unordered_map>
#include <vector>

#include "../../include/wadg.h"

namespace wadg_internal {
void set_error(const std::string &msg);  // wadg_capi.cu
}

struct wadg_mesh {
  int dim = 0;
  std::vector<double> VX;     // [Nv][dim]
  std::vector<int64_t> EToV;  // [K][dim+1], 0-based
  double lo[3] = {0, 0, 0}, hi[3] = {0, 0, 0};
  int64_t flipped = 0;
};

namespace {

int mfail(const std::string &msg) {
  wadg_internal::set_error(msg);
  return WADG_ERR_INVALID;
}

bool read_line(FILE *f, std::string &line) {
  line.clear();
  int c;
  while ((c = fgetc(f)) != EOF) {
    if (c == '\n') return true;
    if (c != '\r') line.push_back((char)c);
  }
  return !line.empty();
}

bool parse_i64(const char *&p, int64_t &v) {
  char *end;
  errno = 0;
  const long long x = strtoll(p, &end, 10);
  if (end == p || errno) return false;
  v = x;
  p = end;
  return true;
}

bool parse_f64(const char *&p, double &v) {
  char *end;
  errno = 0;
  v = strtod(p, &end);
  if (end == p || errno == ERANGE) return false;
  p = end;
  return true;
}

// signed measure of a simplex (twice the area / six times the volume)
double orient(int dim, const double *a, const double *b, const double *c, const double *d) {
  if (dim == 2) return (b[0] - a[0]) * (c[1] - a[1]) - (b[1] - a[1]) * (c[0] - a[0]);
  const double u[3] = {b[0] - a[0], b[1] - a[1], b[2] - a[2]};
  const double v[3] = {c[0] - a[0], c[1] - a[1], c[2] - a[2]};
  const double w[3] = {d[0] - a[0], d[1] - a[1], d[2] - a[2]};
  return u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) +
         u[2] * (v[0] * w[1] - v[1] * w[0]);
}

// face vertices of the reference's elements (euler.c:429-433, 465-470)
const int kFToFV2[3][2] = {{0, 1}, {1, 2}, {2, 0}};
const int kFToFV3[4][3] = {{0, 1, 2}, {0, 1, 3}, {1, 2, 3}, {0, 2, 3}};

}  // namespace

extern "C" {

int wadg_mesh_read_gmsh(const char *path, int dim, wadg_mesh **out) {
  if (!path || !out) return mfail("wadg_mesh_read_gmsh: null argument");
  *out = nullptr;
  if (dim != 2 && dim != 3) return mfail("wadg_mesh_read_gmsh: dim must be 2 or 3");
  FILE *f = fopen(path, "rb");
  if (!f) return mfail(std::string("wadg_mesh_read_gmsh: cannot open ") + path);
  const int nv = dim + 1, want_type = dim == 2 ? 2 : 4;
  std::unordered_map<int64_t, int64_t> node_index;
  std::vector<double> VX;
  std::vector<int64_t> raw;  // element vertices as gmsh node ids
  bool have_format = false, have_nodes = false, have_elements = false;
  std::string line, err;
  while (err.empty() && read_line(f, line)) {
    if (line.rfind("$MeshFormat", 0) == 0) {
      if (!read_line(f, line)) { err = "truncated $MeshFormat"; break; }
      const char *p = line.c_str();
      double version;
      int64_t ftype;
      if (!parse_f64(p, version) || !parse_i64(p, ftype)) { err = "bad $MeshFormat line"; break; }
      if (version < 2.0 || version >= 3.0) { err = "only gmsh 2.x files are read"; break; }
      if (ftype != 0) { err = "binary gmsh files are not read"; break; }
      have_format = true;
    } else if (line.rfind("$Nodes", 0) == 0) {
      if (!read_line(f, line)) { err = "truncated $Nodes"; break; }
      const char *p = line.c_str();
      int64_t n;
      if (!parse_i64(p, n) || n < 0) { err = "bad node count"; break; }
      VX.resize((size_t)n * dim);
      node_index.reserve((size_t)n);
      for (int64_t i = 0; i < n; ++i) {
        if (!read_line(f, line)) { err = "truncated $Nodes"; break; }
        const char *q = line.c_str();
        int64_t id;
        double x[3];
        if (!parse_i64(q, id) || !parse_f64(q, x[0]) || !parse_f64(q, x[1]) || !parse_f64(q, x[2])) {
          err = "bad node line: " + line;
          break;
        }
        if (!node_index.emplace(id, i).second) { err = "duplicate node id"; break; }
        for (int d = 0; d < dim; ++d) VX[(size_t)i * dim + d] = x[d];
      }
      if (!err.empty()) break;
      have_nodes = true;
    } else if (line.rfind("$Elements", 0) == 0) {
      if (!read_line(f, line)) { err = "truncated $Elements"; break; }
      const char *p = line.c_str();
      int64_t n;
      if (!parse_i64(p, n) || n < 0) { err = "bad element count"; break; }
      for (int64_t i = 0; i < n; ++i) {
        if (!read_line(f, line)) { err = "truncated $Elements"; break; }
        const char *q = line.c_str();
        int64_t id, type, ntags, tmp;
        if (!parse_i64(q, id) || !parse_i64(q, type) || !parse_i64(q, ntags) || ntags < 0) {
          err = "bad element line: " + line;
          break;
        }
        if (type != want_type) continue;
        for (int64_t t = 0; t < ntags && err.empty(); ++t)
          if (!parse_i64(q, tmp)) err = "bad element tags: " + line;
        for (int v = 0; v < nv && err.empty(); ++v) {
          if (!parse_i64(q, tmp))
            err = "bad element vertices: " + line;
          else
            raw.push_back(tmp);
        }
        if (!err.empty()) break;
      }
      have_elements = err.empty();
    }
  }
  fclose(f);
  if (err.empty() && !have_format) err = "no $MeshFormat section";
  if (err.empty() && !have_nodes) err = "no $Nodes section";
  if (err.empty() && !have_elements) err = "no $Elements section";
  if (err.empty() && raw.empty()) err = "no elements of the requested dimension";
  if (!err.empty()) return mfail(std::string("wadg_mesh_read_gmsh: ") + path + ": " + err);

  wadg_mesh *m = new wadg_mesh;
  m->dim = dim;
  m->VX = std::move(VX);
  const size_t K = raw.size() / nv;
  m->EToV.resize(raw.size());
  for (size_t i = 0; i < raw.size(); ++i) {
    auto it = node_index.find(raw[i]);
    if (it == node_index.end()) {
      delete m;
      return mfail(std::string("wadg_mesh_read_gmsh: ") + path + ": element refers to a missing node");
    }
    m->EToV[i] = it->second;
  }
  for (size_t k = 0; k < K; ++k) {
    int64_t *e = &m->EToV[k * nv];
    const double *a = &m->VX[(size_t)e[0] * dim], *b = &m->VX[(size_t)e[1] * dim],
                 *c = &m->VX[(size_t)e[2] * dim];
    const double *d = dim == 3 ? &m->VX[(size_t)e[3] * dim] : nullptr;
    const double s = orient(dim, a, b, c, d);
    if (s == 0.0) {
      delete m;
      return mfail(std::string("wadg_mesh_read_gmsh: ") + path + ": degenerate element");
    }
    if (s < 0) {
      std::swap(e[1], e[2]);
      ++m->flipped;
    }
  }
  for (int d = 0; d < dim; ++d) {
    m->lo[d] = HUGE_VAL;
    m->hi[d] = -HUGE_VAL;
  }
  // the periodic box: the bounding box of the elements' vertices
  for (size_t i = 0; i < m->EToV.size(); ++i)
    for (int d = 0; d < dim; ++d) {
      const double x = m->VX[(size_t)m->EToV[i] * dim + d];
      m->lo[d] = fmin(m->lo[d], x);
      m->hi[d] = fmax(m->hi[d], x);
    }
  *out = m;
  return WADG_OK;
}

int wadg_mesh_sizes(const wadg_mesh *m, int *dim, int64_t *Nv, int64_t *K, int64_t *flipped) {
  if (!m) return mfail("wadg_mesh_sizes: null mesh");
  if (dim) *dim = m->dim;
  if (Nv) *Nv = (int64_t)(m->VX.size() / m->dim);
  if (K) *K = (int64_t)(m->EToV.size() / (m->dim + 1));
  if (flipped) *flipped = m->flipped;
  return WADG_OK;
}

int wadg_mesh_get(const wadg_mesh *m, double *VX, int64_t *EToV, double *lo, double *hi) {
  if (!m) return mfail("wadg_mesh_get: null mesh");
  if (VX) memcpy(VX, m->VX.data(), sizeof(double) * m->VX.size());
  if (EToV) memcpy(EToV, m->EToV.data(), sizeof(int64_t) * m->EToV.size());
  if (lo) memcpy(lo, m->lo, sizeof(double) * m->dim);
  if (hi) memcpy(hi, m->hi, sizeof(double) * m->dim);
  return WADG_OK;
}

void wadg_mesh_destroy(wadg_mesh *m) { delete m; }

int wadg_mesh_write_gmsh(const char *path, int dim, int64_t Nv, const double *VX, int64_t K,
                         const int64_t *EToV) {
  if (!path || (Nv > 0 && !VX) || (K > 0 && !EToV) || Nv < 0 || K < 0)
    return mfail("wadg_mesh_write_gmsh: invalid argument");
  if (dim != 2 && dim != 3) return mfail("wadg_mesh_write_gmsh: dim must be 2 or 3");
  FILE *f = fopen(path, "w");
  if (!f) return mfail(std::string("wadg_mesh_write_gmsh: cannot open ") + path);
  const int nv = dim + 1;
  fprintf(f, "$MeshFormat\n2.2 0 8\n$EndMeshFormat\n$Nodes\n%lld\n", (long long)Nv);
  for (int64_t i = 0; i < Nv; ++i)
    fprintf(f, "%lld %.17g %.17g %.17g\n", (long long)(i + 1), VX[i * dim], VX[i * dim + 1],
            dim == 3 ? VX[i * dim + 2] : 0.0);
  fprintf(f, "$EndNodes\n$Elements\n%lld\n", (long long)K);
  for (int64_t k = 0; k < K; ++k) {
    fprintf(f, "%lld %d 2 0 1", (long long)(k + 1), dim == 2 ? 2 : 4);
    for (int v = 0; v < nv; ++v) fprintf(f, " %lld", (long long)(EToV[k * nv + v] + 1));
    fprintf(f, "\n");
  }
  fprintf(f, "$EndElements\n");
  const bool bad = ferror(f) != 0;
  if (fclose(f) != 0 || bad) return mfail(std::string("wadg_mesh_write_gmsh: write error on ") + path);
  return WADG_OK;
}

int wadg_mesh_write_mfem(const char *path, int dim, int64_t K, const double *EToVX,
                         const uint8_t *bface) {
  if (!path || K < 0 || (K > 0 && !EToVX)) return mfail("wadg_mesh_write_mfem: invalid argument");
  if (dim != 2 && dim != 3) return mfail("wadg_mesh_write_mfem: dim must be 2 or 3");
  FILE *f = fopen(path, "w");
  if (!f) return mfail(std::string("wadg_mesh_write_mfem: cannot open ") + path);
  const int nv = dim + 1, nfaces = dim + 1, nfv = dim;
  const int elem_type = dim == 2 ? 2 : 4, face_type = dim == 2 ? 1 : 2;
  fprintf(f, "MFEM mesh v1.0\n\ndimension\n%d\n\nelements\n%lld\n", dim, (long long)K);
  for (int64_t k = 0; k < K; ++k) {
    fprintf(f, "%lld %d", (long long)(k + 1), elem_type);
    for (int v = 0; v < nv; ++v) fprintf(f, " %lld", (long long)(nv * k + v));
    fprintf(f, "\n");
  }
  int64_t nb = 0;
  if (bface)
    for (int64_t i = 0; i < K * nfaces; ++i) nb += bface[i] != 0;
  fprintf(f, "\nboundary\n%lld\n", (long long)nb);
  for (int64_t k = 0; bface && k < K; ++k)
    for (int fc = 0; fc < nfaces; ++fc) {
      if (!bface[k * nfaces + fc]) continue;
      fprintf(f, "%d %d", 1, face_type);
      for (int n = 0; n < nfv; ++n)
        fprintf(f, " %lld", (long long)(nv * k + (dim == 2 ? kFToFV2[fc][n] : kFToFV3[fc][n])));
      fprintf(f, "\n");
    }
  fprintf(f, "vertices\n%lld\n%d\n", (long long)(nv * K), dim);
  for (int64_t k = 0; k < K; ++k)
    for (int v = 0; v < nv; ++v) {
      fprintf(f, "        ");
      for (int d = 0; d < dim; ++d) fprintf(f, " %24.16e", EToVX[(k * nv + v) * dim + d]);
      fprintf(f, "\n");
    }
  const bool bad = ferror(f) != 0;
  if (fclose(f) != 0 || bad) return mfail(std::string("wadg_mesh_write_mfem: write error on ") + path);
  return WADG_OK;
}

}  // extern "C"
