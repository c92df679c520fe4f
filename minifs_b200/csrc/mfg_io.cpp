// FlowStar files: the binary grid (ReadMFlowGrid_binary,
// src/Kernels/load_grid.cpp:129-273) and the boundary-condition table
// (ReadMFlowBoundaryCondition, :282-314), read and written on the host.
//
// The reader keeps the reference's one transformation of the file's arrays
// (faces whose first cell is a boundary are flipped) and its boundary-face
// count; it checks what the reference takes on trust (sizes, truncation,
// trailing bytes) and reports MFG_ERR_IO instead of reading past the data.
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

#include "mfgpu.h"

namespace {

struct File {
  FILE *fp = nullptr;
  explicit File(FILE *f) : fp(f) {}
  ~File() {
    if (fp) fclose(fp);
  }
};

template <typename T>
bool read_n(FILE *fp, T *dst, int64_t n) {
  if (n <= 0) return true;
  return fread(dst, sizeof(T), (size_t)n, fp) == (size_t)n;
}

template <typename T>
bool write_n(FILE *fp, const T *src, int64_t n) {
  if (n <= 0) return true;
  return src && fwrite(src, sizeof(T), (size_t)n, fp) == (size_t)n;
}

template <typename T>
T *alloc_n(int64_t n) {
  return static_cast<T *>(std::malloc(sizeof(T) * (size_t)(n > 0 ? n : 1)));
}

void free_arrays(mfg_mfl *g) {
  std::free(g->x);
  std::free(g->y);
  std::free(g->z);
  std::free(g->nnpf);
  std::free(g->f2n);
  std::free(g->f2c);
  std::free(g->nbz);
  std::free(g->nbf);
  std::free(g->nbsn);
  std::free(g->nbzn);
  std::free(g->nbrn);
}

int64_t remaining(FILE *fp) {
  const long here = ftell(fp);
  if (here < 0 || fseek(fp, 0, SEEK_END) != 0) return -1;
  const long end = ftell(fp);
  if (end < 0 || fseek(fp, here, SEEK_SET) != 0) return -1;
  return (int64_t)end - here;
}

int read_impl(FILE *fp, mfg_mfl *g) {
  int32_t head[3];
  if (!read_n(fp, head, 3)) return MFG_ERR_IO;
  const int32_t N = head[0], F = head[1], C = head[2];
  if (N < 0 || F < 0 || C < 0) return MFG_ERR_IO;
  // everything up to f2n must be in the file before anything is allocated
  const int64_t left = remaining(fp);
  if (left < 0 || left < 24 * (int64_t)N + 4 * (int64_t)F) return MFG_ERR_IO;
  g->n_node = N;
  g->n_face = F;
  g->n_cell = C;
  if (!(g->x = alloc_n<double>(N)) || !(g->y = alloc_n<double>(N)) ||
      !(g->z = alloc_n<double>(N)) || !(g->nnpf = alloc_n<int32_t>(F)))
    return MFG_ERR_NOMEM;
  if (!read_n(fp, g->x, N) || !read_n(fp, g->y, N) || !read_n(fp, g->z, N) ||
      !read_n(fp, g->nnpf, F))
    return MFG_ERR_IO;
  // facnod (:192-198)
  std::vector<int64_t> ptr((size_t)F + 1, 0);
  for (int32_t i = 0; i < F; i++) {
    if (g->nnpf[i] < 1) return MFG_ERR_IO;
    ptr[i + 1] = ptr[i] + g->nnpf[i];
  }
  const int64_t L = ptr[F];
  if (L > INT32_MAX || remaining(fp) < 4 * (L + 2 * (int64_t)F)) return MFG_ERR_IO;
  if (!(g->f2n = alloc_n<int32_t>(L)) || !(g->f2c = alloc_n<int32_t>(2 * (int64_t)F)))
    return MFG_ERR_NOMEM;
  if (!read_n(fp, g->f2n, L) || !read_n(fp, g->f2c, 2 * (int64_t)F)) return MFG_ERR_IO;
  // boundary faces (:209-229): a boundary on the left is moved to the right,
  // the node order reversed behind the first node to keep the normal outward
  int32_t nb = 0;
  for (int32_t i = 0; i < F; i++) {
    int32_t *c = g->f2c + 2 * (int64_t)i;
    if (c[0] < 0) {
      int32_t *a = g->f2n + ptr[i] + 1, *b = g->f2n + ptr[i + 1] - 1;
      for (; a < b; a++, b--) {
        const int32_t t = *a;
        *a = *b;
        *b = t;
      }
      const int32_t t = c[0];
      c[0] = c[1];
      c[1] = t;
      nb++;
    } else if (c[1] < 0) {
      nb++;
    }
  }
  g->n_bface = nb;
  // interface block (:232-263)
  const int64_t tail = remaining(fp);
  if (tail < 0) return MFG_ERR_IO;
  if (tail == 0) return MFG_OK;  // no block: no interfaces
  int32_t ni = 0, nn = 0;
  if (!read_n(fp, &ni, 1) || ni < 0 || remaining(fp) < 8 * (int64_t)ni + 4) return MFG_ERR_IO;
  g->n_iface = ni;
  if (!(g->nbz = alloc_n<int32_t>(ni)) || !(g->nbf = alloc_n<int32_t>(ni))) return MFG_ERR_NOMEM;
  if (!read_n(fp, g->nbz, ni) || !read_n(fp, g->nbf, ni) || !read_n(fp, &nn, 1) || nn < 0 ||
      remaining(fp) < 12 * (int64_t)nn)
    return MFG_ERR_IO;
  g->n_inode = nn;
  if (!(g->nbsn = alloc_n<int32_t>(nn)) || !(g->nbzn = alloc_n<int32_t>(nn)) ||
      !(g->nbrn = alloc_n<int32_t>(nn)))
    return MFG_ERR_NOMEM;
  if (!read_n(fp, g->nbsn, nn) || !read_n(fp, g->nbzn, nn) || !read_n(fp, g->nbrn, nn))
    return MFG_ERR_IO;
  return remaining(fp) == 0 ? MFG_OK : MFG_ERR_IO;
}

}  // namespace

extern "C" {

int mfg_mfl_read(const char *path, mfg_mfl **out) {
  if (!path || !out) return MFG_ERR_INVALID;
  *out = nullptr;
  File f(fopen(path, "rb"));
  if (!f.fp) return MFG_ERR_IO;
  mfg_mfl *g = new (std::nothrow) mfg_mfl();
  if (!g) return MFG_ERR_NOMEM;
  const int rc = read_impl(f.fp, g);
  if (rc != MFG_OK) {
    free_arrays(g);
    delete g;
    return rc;
  }
  *out = g;
  return MFG_OK;
}

int mfg_mfl_write(const char *path, const mfg_mfl *g) {
  if (!path || !g || g->n_node < 0 || g->n_face < 0 || g->n_cell < 0 || g->n_iface < 0 ||
      g->n_inode < 0)
    return MFG_ERR_INVALID;
  int64_t L = 0;
  for (int32_t i = 0; i < g->n_face; i++) {
    if (!g->nnpf || g->nnpf[i] < 1) return MFG_ERR_INVALID;
    L += g->nnpf[i];
  }
  File f(fopen(path, "wb"));
  if (!f.fp) return MFG_ERR_IO;
  const int32_t head[3] = {g->n_node, g->n_face, g->n_cell};
  const int32_t ni = g->n_iface, nn = g->n_inode;
  const bool ok = write_n(f.fp, head, 3) && write_n(f.fp, g->x, g->n_node) &&
                  write_n(f.fp, g->y, g->n_node) && write_n(f.fp, g->z, g->n_node) &&
                  write_n(f.fp, g->nnpf, g->n_face) && write_n(f.fp, g->f2n, L) &&
                  write_n(f.fp, g->f2c, 2 * (int64_t)g->n_face) && write_n(f.fp, &ni, 1) &&
                  write_n(f.fp, g->nbz, ni) && write_n(f.fp, g->nbf, ni) &&
                  write_n(f.fp, &nn, 1) && write_n(f.fp, g->nbsn, nn) &&
                  write_n(f.fp, g->nbzn, nn) && write_n(f.fp, g->nbrn, nn);
  if (!ok) return MFG_ERR_IO;
  if (fflush(f.fp) != 0) return MFG_ERR_IO;
  return MFG_OK;
}

int mfg_mfl_free(mfg_mfl *g) {
  if (!g) return MFG_ERR_INVALID;
  free_arrays(g);
  delete g;
  return MFG_OK;
}

int mfg_bc_read(const char *path, int32_t cap, int32_t *n_patch, int32_t *patch_id,
                int32_t *type) {
  if (!path || !n_patch || cap < 0 || (cap > 0 && (!patch_id || !type))) return MFG_ERR_INVALID;
  File f(fopen(path, "r"));
  if (!f.fp) return MFG_ERR_IO;
  int n = 0;
  if (fscanf(f.fp, "%d", &n) != 1 || n < 0) return MFG_ERR_IO;
  *n_patch = n;
  if (n > cap) return MFG_ERR_INVALID;
  for (int i = 0; i < n; i++) {
    int pid = 0, t = 0;
    if (fscanf(f.fp, "%d %d", &pid, &t) != 2) return MFG_ERR_IO;
    patch_id[i] = pid;
    type[i] = t;
  }
  return MFG_OK;
}

// Checkpoint file: "MFGCKPT1", int64 n_cell, int64 n (cells + ghosts), int32
// iter_done, int32 0, double dt_max, double dt_min, double q[5 n].
static const char kCkptMagic[8] = {'M', 'F', 'G', 'C', 'K', 'P', 'T', '1'};

int mfg_checkpoint_write(const char *path, int64_t n_cell, int64_t n, int32_t iter_done,
                         double dt_max, double dt_min, const double *q) {
  if (!path || n_cell < 0 || n < n_cell || iter_done < 0 || (n > 0 && !q))
    return MFG_ERR_INVALID;
  File f(fopen(path, "wb"));
  if (!f.fp) return MFG_ERR_IO;
  const int32_t pad = 0;
  if (!write_n(f.fp, kCkptMagic, 8) || !write_n(f.fp, &n_cell, 1) || !write_n(f.fp, &n, 1) ||
      !write_n(f.fp, &iter_done, 1) || !write_n(f.fp, &pad, 1) || !write_n(f.fp, &dt_max, 1) ||
      !write_n(f.fp, &dt_min, 1) || !write_n(f.fp, q, 5 * n))
    return MFG_ERR_IO;
  if (fflush(f.fp) != 0) return MFG_ERR_IO;
  return MFG_OK;
}

int mfg_checkpoint_read(const char *path, int64_t n_cell, int64_t n, int32_t *iter_done,
                        double *dt_max, double *dt_min, double *q) {
  if (!path || n_cell < 0 || n < n_cell || !iter_done || !dt_max || !dt_min || (n > 0 && !q))
    return MFG_ERR_INVALID;
  File f(fopen(path, "rb"));
  if (!f.fp) return MFG_ERR_IO;
  char magic[8];
  int64_t fc = -1, fn = -1;
  int32_t it = -1, pad = 0;
  double mx = 0.0, mn = 0.0;
  if (!read_n(f.fp, magic, 8) || std::memcmp(magic, kCkptMagic, 8) != 0 ||
      !read_n(f.fp, &fc, 1) || !read_n(f.fp, &fn, 1) || !read_n(f.fp, &it, 1) ||
      !read_n(f.fp, &pad, 1) || !read_n(f.fp, &mx, 1) || !read_n(f.fp, &mn, 1))
    return MFG_ERR_IO;
  if (fc != n_cell || fn != n || it < 0) return MFG_ERR_INVALID;  // another grid
  if (remaining(f.fp) != 40 * n) return MFG_ERR_IO;
  if (!read_n(f.fp, q, 5 * n)) return MFG_ERR_IO;
  *iter_done = it;
  *dt_max = mx;
  *dt_min = mn;
  return MFG_OK;
}

int mfg_bc_write(const char *path, int32_t n_patch, const int32_t *patch_id,
                 const int32_t *type) {
  if (!path || n_patch < 0 || (n_patch > 0 && (!patch_id || !type))) return MFG_ERR_INVALID;
  File f(fopen(path, "w"));
  if (!f.fp) return MFG_ERR_IO;
  if (fprintf(f.fp, "%d\n", n_patch) < 0) return MFG_ERR_IO;
  for (int32_t i = 0; i < n_patch; i++)
    if (fprintf(f.fp, "%d %d\n", patch_id[i], type[i]) < 0) return MFG_ERR_IO;
  if (fflush(f.fp) != 0) return MFG_ERR_IO;
  return MFG_OK;
}

}  // extern "C"
