// Seeded finite-volume systems on hexahedral boxes in SFR3D's sparse layouts.
// Host-only code (libsfr3d_systems.so).  Conventions and layouts are listed
// in include/sfr3d_systems.h with the reference lines they follow.
#include "sfr3d_systems.h"

#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <new>
#include <vector>

namespace {

// splitmix64 (Steele, Lea, Flood 2014) seeding xoshiro256** (Blackman, Vigna
// 2018): both published generators, written here from their definitions.
uint64_t splitmix64(uint64_t &state) {
  uint64_t z = (state += 0x9E3779B97F4A7C15ULL);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
  return z ^ (z >> 31);
}

class Rng {
 public:
  explicit Rng(uint64_t seed) {
    uint64_t st = seed;
    for (auto &w : s_) w = splitmix64(st);
  }
  uint64_t next() {
    const uint64_t result = rotl(s_[1] * 5, 7) * 9;
    const uint64_t t = s_[1] << 17;
    s_[2] ^= s_[0];
    s_[3] ^= s_[1];
    s_[1] ^= s_[2];
    s_[0] ^= s_[3];
    s_[2] ^= t;
    s_[3] = rotl(s_[3], 45);
    return result;
  }
  // uniform on [0, 1) with 53 random bits
  double uniform() { return static_cast<double>(next() >> 11) * 0x1.0p-53; }
  double uniform(double a, double b) { return a + (b - a) * uniform(); }
  // Box-Muller on (0,1] x [0,1)
  double normal() {
    if (has_spare_) {
      has_spare_ = false;
      return spare_;
    }
    const double u1 = 1.0 - uniform();
    const double u2 = uniform();
    const double rad = std::sqrt(-2.0 * std::log(u1));
    const double ang = 6.283185307179586476925 * u2;
    spare_ = rad * std::sin(ang);
    has_spare_ = true;
    return rad * std::cos(ang);
  }
  uint64_t below(uint64_t n) { return next() % n; }

 private:
  static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  uint64_t s_[4];
  bool has_spare_ = false;
  double spare_ = 0.0;
};

struct Vec3 {
  double x, y, z;
};
inline Vec3 operator-(Vec3 a, Vec3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline Vec3 operator+(Vec3 a, Vec3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline Vec3 operator*(double s, Vec3 a) { return {s * a.x, s * a.y, s * a.z}; }
inline double dot(Vec3 a, Vec3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double norm(Vec3 a) { return std::sqrt(dot(a, a)); }
inline Vec3 cross(Vec3 a, Vec3 b) {
  return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x};
}

constexpr int kFaces = 6;  // face order of every cell: x-, x+, y-, y+, z-, z+

struct System {
  sfr_sys_params p{};
  int32_t neq = 0;
  bool unsym = false;
  double velocity_scale = 0.0;
  // per equation (row, new numbering), per face slot
  std::vector<int32_t> nb;    // neighbour equation or -1 on the boundary
  std::vector<double> off;    // A(row, nb) ; -0.0 on boundary slots
  std::vector<double> diag;   // A(row, row)
  std::vector<double> rhs;    // nrhs * neq
  std::vector<int32_t> eq_of_cell;
  int32_t nnz_full = 0, nnz_lower = 0, bandwidth = 0;
  // the mesh itself, kept for the export in the reference's mesh arrays
  std::vector<Vec3> node, centre;  // vertices; cell centres (natural cell id)
  std::vector<double> volume, kappa;
};

// ---------------------------------------------------------------- RCM ----
// Reverse Cuthill-McKee (Cuthill & McKee 1969; George & Liu 1981): a
// pseudo-peripheral root from repeated rooted level structures, breadth-first
// numbering with neighbours taken by increasing degree, then reversal.

// Rooted level structure of the component of `root`: queue[0..*size) in BFS
// order, the deepest level starting at *last_begin.  Returns the depth.
int rooted_levels(int32_t root, const int32_t *xadj, const int32_t *adj,
                  std::vector<int32_t> &level, std::vector<int32_t> &queue,
                  int32_t *size, int32_t *last_begin) {
  int32_t head = 0, tail = 0, lb = 0;
  int depth = 0;
  queue[tail++] = root;
  level[root] = 0;
  while (head < tail) {
    const int32_t u = queue[head++];
    for (int32_t k = xadj[u]; k < xadj[u + 1]; ++k) {
      const int32_t v = adj[k];
      if (level[v] < 0) {
        level[v] = level[u] + 1;
        if (level[v] > depth) {
          depth = level[v];
          lb = tail;
        }
        queue[tail++] = v;
      }
    }
  }
  for (int32_t i = 0; i < tail; ++i) level[queue[i]] = -1;
  *size = tail;
  *last_begin = lb;
  return depth;
}

}  // namespace

extern "C" int sfr_rcm(int32_t n, const int32_t *xadj, const int32_t *adj,
                       int32_t *perm) {
  if (n < 0 || !xadj || (!adj && n > 0 && xadj[n] > 0) || (!perm && n > 0)) return -1;
  for (int32_t i = 0; i < n; ++i) {
    if (xadj[i + 1] < xadj[i]) return -1;
    for (int32_t k = xadj[i]; k < xadj[i + 1]; ++k)
      if (adj[k] < 0 || adj[k] >= n) return -1;
  }
  std::vector<int32_t> deg(n);
  for (int32_t i = 0; i < n; ++i) deg[i] = xadj[i + 1] - xadj[i];
  std::vector<int32_t> level(n, -1), queue(n);
  std::vector<char> numbered(n, 0);
  std::vector<int32_t> order;
  order.reserve(n);
  std::vector<int32_t> nbuf;
  int32_t scan = 0;
  while (static_cast<int32_t>(order.size()) < n) {
    // a new component starts at its unnumbered node of least degree
    while (scan < n && numbered[scan]) ++scan;
    int32_t start = scan;
    for (int32_t i = scan; i < n; ++i)
      if (!numbered[i] && deg[i] < deg[start]) start = i;
    // pseudo-peripheral root
    int32_t root = start, size = 0, lb = 0;
    int depth = rooted_levels(root, xadj, adj, level, queue, &size, &lb);
    for (;;) {
      int32_t cand = queue[lb];
      for (int32_t i = lb; i < size; ++i) {
        const int32_t v = queue[i];
        if (deg[v] < deg[cand] || (deg[v] == deg[cand] && v < cand)) cand = v;
      }
      int32_t size2 = 0, lb2 = 0;
      const int depth2 = rooted_levels(cand, xadj, adj, level, queue, &size2, &lb2);
      if (depth2 <= depth) break;
      root = cand;
      depth = depth2;
      size = size2;
      lb = lb2;
    }
    // Cuthill-McKee numbering of the component from the root
    const size_t first = order.size();
    order.push_back(root);
    numbered[root] = 1;
    for (size_t head = first; head < order.size(); ++head) {
      const int32_t u = order[head];
      nbuf.clear();
      for (int32_t k = xadj[u]; k < xadj[u + 1]; ++k) {
        const int32_t v = adj[k];
        if (!numbered[v]) {
          numbered[v] = 1;
          nbuf.push_back(v);
        }
      }
      std::sort(nbuf.begin(), nbuf.end(), [&](int32_t a, int32_t b) {
        return deg[a] != deg[b] ? deg[a] < deg[b] : a < b;
      });
      order.insert(order.end(), nbuf.begin(), nbuf.end());
    }
  }
  for (int32_t i = 0; i < n; ++i) perm[i] = order[n - 1 - i];
  return 0;
}

namespace {

inline int64_t node_id(int i, int j, int k, int nx, int ny) {
  return static_cast<int64_t>(i) +
         static_cast<int64_t>(nx + 1) *
             (static_cast<int64_t>(j) + static_cast<int64_t>(ny + 1) * k);
}

// The four vertices of the face at node-plane `pl` of axis `ax` spanning the
// cell (u, w) of the two other axes, ordered so that
// 0.5 (v2 - v0) x (v3 - v1) points along +axis.
void face_vertices(const std::vector<Vec3> &node, int nx, int ny, int ax, int pl, int u, int w,
                   Vec3 v[4]) {
  if (ax == 0) {  // x-face: i = pl, j = u, k = w
    v[0] = node[node_id(pl, u, w, nx, ny)];
    v[1] = node[node_id(pl, u + 1, w, nx, ny)];
    v[2] = node[node_id(pl, u + 1, w + 1, nx, ny)];
    v[3] = node[node_id(pl, u, w + 1, nx, ny)];
  } else if (ax == 1) {  // y-face: j = pl, k = u, i = w
    v[0] = node[node_id(w, pl, u, nx, ny)];
    v[1] = node[node_id(w, pl, u + 1, nx, ny)];
    v[2] = node[node_id(w + 1, pl, u + 1, nx, ny)];
    v[3] = node[node_id(w + 1, pl, u, nx, ny)];
  } else {  // z-face: k = pl, i = u, j = w
    v[0] = node[node_id(u, w, pl, nx, ny)];
    v[1] = node[node_id(u + 1, w, pl, nx, ny)];
    v[2] = node[node_id(u + 1, w + 1, pl, nx, ny)];
    v[3] = node[node_id(u, w + 1, pl, nx, ny)];
  }
}

// the cell on the + side of node-plane pl (index pl along ax)
inline int32_t plus_cell(int nx, int ny, int ax, int pl, int u, int w) {
  int i, j, k;
  if (ax == 0) { i = pl; j = u; k = w; }
  else if (ax == 1) { j = pl; k = u; i = w; }
  else { k = pl; i = u; j = w; }
  return i + nx * (j + ny * k);
}

// extents (u, w) of the faces of axis ax
inline void face_span(int nx, int ny, int nz, int ax, int *nu, int *nw) {
  if (ax == 0) { *nu = ny; *nw = nz; }
  else if (ax == 1) { *nu = nz; *nw = nx; }
  else { *nu = nx; *nw = ny; }
}

bool valid(const sfr_sys_params &p) {
  if (p.kind != SFR_SYS_DIFFUSION && p.kind != SFR_SYS_CONVDIFF) return false;
  if (p.nx < 1 || p.ny < 1 || p.nz < 1) return false;
  const double cells = static_cast<double>(p.nx) * p.ny * p.nz;
  if (cells > 2.0e8) return false;
  if (!(p.lx > 0 && p.ly > 0 && p.lz > 0)) return false;
  if (p.jitter < 0 || p.jitter >= 0.5) return false;
  if (p.log10k_hi < p.log10k_lo) return false;
  if (p.nrhs < 0 || p.nrhs > 64) return false;
  if (p.kind == SFR_SYS_CONVDIFF && (p.nu <= 0 || p.dt <= 0 || p.peclet < 0))
    return false;
  return true;
}

System *build(const sfr_sys_params &p) {
  auto *s = new (std::nothrow) System;
  if (!s) return nullptr;
  s->p = p;
  const int nx = p.nx, ny = p.ny, nz = p.nz;
  const int32_t ncell = nx * ny * nz;
  s->neq = ncell;
  s->unsym = p.kind == SFR_SYS_CONVDIFF;
  const double hx = p.lx / nx, hy = p.ly / ny, hz = p.lz / nz;

  // ---- nodes (jittered inside, boundary nodes stay on their faces)
  const int64_t nnode = static_cast<int64_t>(nx + 1) * (ny + 1) * (nz + 1);
  std::vector<Vec3> node(nnode);
  Rng rng_geo(p.seed ^ 0x6A09E667F3BCC908ULL);
  for (int k = 0; k <= nz; ++k)
    for (int j = 0; j <= ny; ++j)
      for (int i = 0; i <= nx; ++i) {
        Vec3 c{i * hx, j * hy, k * hz};
        if (p.jitter > 0) {
          const double dx = rng_geo.uniform(-p.jitter, p.jitter);
          const double dy = rng_geo.uniform(-p.jitter, p.jitter);
          const double dz = rng_geo.uniform(-p.jitter, p.jitter);
          if (i > 0 && i < nx) c.x += dx * hx;
          if (j > 0 && j < ny) c.y += dy * hy;
          if (k > 0 && k < nz) c.z += dz * hz;
        }
        node[node_id(i, j, k, nx, ny)] = c;
      }

  // ---- cells: centre = mean of the 8 vertices, volume by 6 tetrahedra
  std::vector<Vec3> centre(ncell);
  std::vector<double> volume(ncell);
  std::vector<double> kappa(ncell);
  Rng rng_k(p.seed ^ 0xBB67AE8584CAA73BULL);
  for (int k = 0; k < nz; ++k)
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        const int32_t c = i + nx * (j + ny * k);
        Vec3 v[8];
        for (int q = 0; q < 8; ++q)
          v[q] = node[node_id(i + (q & 1), j + ((q >> 1) & 1), k + (q >> 2), nx, ny)];
        Vec3 m{0, 0, 0};
        for (auto &q : v) m = m + q;
        centre[c] = 0.125 * m;
        // volume from the divergence theorem would need the faces; a
        // six-tetrahedra split along the 0-7 diagonal is exact for the
        // trilinear cell when faces are planar and close otherwise
        static const int tets[6][2] = {{1, 3}, {3, 2}, {2, 6}, {6, 4}, {4, 5}, {5, 1}};
        double vol = 0;
        for (auto &t : tets) {
          const Vec3 a = v[t[0]] - v[0], b = v[t[1]] - v[0], d = v[7] - v[0];
          vol += dot(cross(a, b), d) / 6.0;
        }
        volume[c] = std::fabs(vol);
        const double e = (p.log10k_hi > p.log10k_lo)
                             ? rng_k.uniform(p.log10k_lo, p.log10k_hi)
                             : p.log10k_lo;
        kappa[c] = std::pow(10.0, e);
      }

  // ---- faces: per cell, neighbour (natural id), off-diagonal, sP parts
  std::vector<int32_t> nb_nat(static_cast<size_t>(ncell) * kFaces, -1);
  std::vector<double> a_nat(static_cast<size_t>(ncell) * kFaces, 0.0);
  std::vector<double> sP(ncell, 0.0);

  // face geometry of the face at node-plane `pl` of axis `ax` spanning the
  // cell (u, w) of the two other axes; area vector points along +axis
  auto face = [&](int ax, int pl, int u, int w, Vec3 *S, Vec3 *xf) {
    Vec3 v[4];
    face_vertices(node, nx, ny, ax, pl, u, w, v);
    *S = 0.5 * cross(v[2] - v[0], v[3] - v[1]);
    *xf = 0.25 * (v[0] + v[1] + v[2] + v[3]);
  };

  // convective face flux in +axis direction for unit velocity scale, from the
  // exact face integral of u = (sin x cos y cos z, -cos x sin y cos z, 0)
  auto flux_unit = [&](int ax, int pl, int u, int w) -> double {
    if (ax == 0) {
      const double x = pl * hx, y0 = u * hy, y1 = (u + 1) * hy, z0 = w * hz,
                   z1 = (w + 1) * hz;
      return std::sin(x) * (std::sin(y1) - std::sin(y0)) * (std::sin(z1) - std::sin(z0));
    }
    if (ax == 1) {
      const double y = pl * hy, z0 = u * hz, z1 = (u + 1) * hz, x0 = w * hx,
                   x1 = (w + 1) * hx;
      return -(std::sin(x1) - std::sin(x0)) * std::sin(y) * (std::sin(z1) - std::sin(z0));
    }
    return 0.0;
  };

  const int dims[3] = {nx, ny, nz};
  auto cell_of = [&](int ax, int pl, int u, int w) -> int32_t {
    return plus_cell(nx, ny, ax, pl, u, w);
  };
  auto span = [&](int ax, int *nu, int *nw) { face_span(nx, ny, nz, ax, nu, nw); };

  // Peclet scaling: U = peclet / max_f(|F_unit| / D_f) over interior faces
  double U = 0.0;
  if (p.kind == SFR_SYS_CONVDIFF) {
    double worst = 0.0;
    for (int ax = 0; ax < 3; ++ax) {
      int nu, nw;
      span(ax, &nu, &nw);
      for (int pl = 1; pl < dims[ax]; ++pl)
        for (int w = 0; w < nw; ++w)
          for (int u = 0; u < nu; ++u) {
            Vec3 S, xf;
            face(ax, pl, u, w, &S, &xf);
            const int32_t cp = cell_of(ax, pl, u, w);
            const int32_t cm = cell_of(ax, pl - 1, u, w);
            const double D = p.nu * norm(S) / norm(centre[cp] - centre[cm]);
            worst = std::max(worst, std::fabs(flux_unit(ax, pl, u, w)) / D);
          }
    }
    U = worst > 0 ? p.peclet / worst : 0.0;
    s->velocity_scale = U;
  }

  for (int ax = 0; ax < 3; ++ax) {
    int nu, nw;
    span(ax, &nu, &nw);
    for (int pl = 0; pl <= dims[ax]; ++pl)
      for (int w = 0; w < nw; ++w)
        for (int u = 0; u < nu; ++u) {
          Vec3 S, xf;
          face(ax, pl, u, w, &S, &xf);
          const double area = norm(S);
          const bool has_minus = pl > 0, has_plus = pl < dims[ax];
          const int32_t cm = has_minus ? cell_of(ax, pl - 1, u, w) : -1;
          const int32_t cp = has_plus ? cell_of(ax, pl, u, w) : -1;
          const int fm = 2 * ax + 1;  // face slot of the face in cell cm (+ side)
          const int fp = 2 * ax;      // face slot in cell cp (- side)
          if (has_minus && has_plus) {
            const Vec3 xi = centre[cp] - centre[cm];
            const double d = norm(xi);
            if (p.kind == SFR_SYS_DIFFUSION) {
              const Vec3 e = (1.0 / d) * xi;
              const double dPf = dot(xf - centre[cm], e);
              const double dfN = dot(centre[cp] - xf, e);
              const double alpha = dPf / (dPf + dfN);
              const double kf = 1.0 / (alpha / kappa[cm] + (1.0 - alpha) / kappa[cp]);
              const double a = kf * area / d;
              a_nat[static_cast<size_t>(cm) * kFaces + fm] = a;
              a_nat[static_cast<size_t>(cp) * kFaces + fp] = a;
            } else {
              const double D = p.nu * area / d;
              const double F = U * flux_unit(ax, pl, u, w);  // + axis direction
              // outward flux from cm is +F, from cp is -F
              a_nat[static_cast<size_t>(cm) * kFaces + fm] = D + std::max(-F, 0.0);
              a_nat[static_cast<size_t>(cp) * kFaces + fp] = D + std::max(F, 0.0);
              sP[cm] += F;
              sP[cp] += -F;
            }
            nb_nat[static_cast<size_t>(cm) * kFaces + fm] = cp;
            nb_nat[static_cast<size_t>(cp) * kFaces + fp] = cm;
          } else {
            const int32_t c = has_plus ? cp : cm;
            const int side_bit = has_plus ? (1 << (2 * ax)) : (1 << (2 * ax + 1));
            if (p.dirichlet_faces & side_bit) {
              const double dPf = norm(xf - centre[c]);
              const double k = p.kind == SFR_SYS_DIFFUSION ? kappa[c] : p.nu;
              sP[c] += k * area / dPf;
            }
          }
        }
  }
  if (p.kind == SFR_SYS_CONVDIFF)
    for (int32_t c = 0; c < ncell; ++c) sP[c] += volume[c] / p.dt;

  // ---- numbering: optional random permutation, then RCM
  std::vector<int32_t> label(ncell);
  for (int32_t c = 0; c < ncell; ++c) label[c] = c;
  if (p.permute) {
    Rng rng_p(p.seed ^ 0x3C6EF372FE94F82BULL);
    for (int32_t i = ncell - 1; i > 0; --i) {
      const int32_t j = static_cast<int32_t>(rng_p.below(static_cast<uint64_t>(i) + 1));
      std::swap(label[i], label[j]);
    }
  }
  std::vector<int32_t> cell_of_label(ncell);
  for (int32_t c = 0; c < ncell; ++c) cell_of_label[label[c]] = c;
  std::vector<int32_t> eq_of_label(ncell);
  if (p.rcm) {
    std::vector<int32_t> xadj(ncell + 1, 0), adj;
    adj.reserve(static_cast<size_t>(ncell) * kFaces);
    std::vector<int32_t> tmp;
    for (int32_t l = 0; l < ncell; ++l) {
      const int32_t c = cell_of_label[l];
      tmp.clear();
      for (int f = 0; f < kFaces; ++f) {
        const int32_t n = nb_nat[static_cast<size_t>(c) * kFaces + f];
        if (n >= 0) tmp.push_back(label[n]);
      }
      std::sort(tmp.begin(), tmp.end());
      adj.insert(adj.end(), tmp.begin(), tmp.end());
      xadj[l + 1] = static_cast<int32_t>(adj.size());
    }
    std::vector<int32_t> perm(ncell);
    sfr_rcm(ncell, xadj.data(), adj.data(), perm.data());
    for (int32_t e = 0; e < ncell; ++e) eq_of_label[perm[e]] = e;
  } else {
    for (int32_t l = 0; l < ncell; ++l) eq_of_label[l] = l;
  }
  s->eq_of_cell.resize(ncell);
  for (int32_t c = 0; c < ncell; ++c) s->eq_of_cell[c] = eq_of_label[label[c]];

  // ---- rows in equation order
  s->nb.assign(static_cast<size_t>(ncell) * kFaces, -1);
  s->off.assign(static_cast<size_t>(ncell) * kFaces, -0.0);
  s->diag.assign(ncell, 0.0);
  int32_t nnz = 0, band = 0;
  for (int32_t c = 0; c < ncell; ++c) {
    const int32_t r = s->eq_of_cell[c];
    double an = 0.0;
    for (int f = 0; f < kFaces; ++f) {
      const size_t q = static_cast<size_t>(c) * kFaces + f;
      an += a_nat[q];
      const int32_t n = nb_nat[q];
      if (n >= 0) {
        const int32_t col = s->eq_of_cell[n];
        s->nb[static_cast<size_t>(r) * kFaces + f] = col;
        s->off[static_cast<size_t>(r) * kFaces + f] = -a_nat[q];
        ++nnz;
        band = std::max(band, std::abs(col - r));
      }
    }
    s->diag[r] = sP[c] + an;
  }
  s->nnz_full = nnz;
  s->nnz_lower = nnz / 2;
  s->bandwidth = band;

  // ---- right-hand sides, drawn in equation order
  s->rhs.resize(static_cast<size_t>(p.nrhs) * ncell);
  Rng rng_b(p.seed ^ 0xA54FF53A5F1D36F1ULL);
  for (auto &v : s->rhs) v = p.rhs_normal ? rng_b.normal() : rng_b.uniform(-1.0, 1.0);
  s->node = std::move(node);
  s->centre = std::move(centre);
  s->volume = std::move(volume);
  s->kappa = std::move(kappa);
  return s;
}

int64_t face_count(const sfr_sys_params &p) {
  return static_cast<int64_t>(p.nx + 1) * p.ny * p.nz + static_cast<int64_t>(p.ny + 1) * p.nz * p.nx +
         static_cast<int64_t>(p.nz + 1) * p.nx * p.ny;
}

inline Vec3 unit(Vec3 a) { return (1.0 / norm(a)) * a; }

// The box as the reference's mesh arrays (the inputs of systFormDif,
// CellLoop.c:285-311).  Faces are numbered axis by axis, node-plane by
// node-plane, in the order build() visits them.  The owner of a face is its
// minus-side cell (the plus-side cell for a face on a minus boundary); the
// face vectors point out of the owner, and a cell that is not the owner takes
// them negated (OWNER, CellLoop.c:376-388).
void export_mesh(const System &s, const sfr_sys_mesh_t &m) {
  const int nx = s.p.nx, ny = s.p.ny, nz = s.p.nz;
  const int32_t ncell = nx * ny * nz;
  const int dims[3] = {nx, ny, nz};
  for (int32_t c = 0; c < ncell; ++c) {
    m.nviz[c] = kFaces;
    m.volume[c] = s.volume[c];
    m.cdiff[c] = s.kappa[c];
    m.id[c] = s.eq_of_cell[c] + 1;
  }
  int64_t f = 0;
  for (int ax = 0; ax < 3; ++ax) {
    int nu, nw;
    face_span(nx, ny, nz, ax, &nu, &nw);
    for (int pl = 0; pl <= dims[ax]; ++pl)
      for (int w = 0; w < nw; ++w)
        for (int u = 0; u < nu; ++u, ++f) {
          Vec3 v[4];
          face_vertices(s.node, nx, ny, ax, pl, u, w, v);
          const Vec3 S = 0.5 * cross(v[2] - v[0], v[3] - v[1]);
          const Vec3 xm = 0.25 * (v[0] + v[1] + v[2] + v[3]);
          const bool has_minus = pl > 0, has_plus = pl < dims[ax];
          const int32_t cm = has_minus ? plus_cell(nx, ny, ax, pl - 1, u, w) : -1;
          const int32_t cp = has_plus ? plus_cell(nx, ny, ax, pl, u, w) : -1;
          const int32_t own = has_minus ? cm : cp;
          const int32_t nbr = has_minus && has_plus ? cp : -1;
          const double area = norm(S);
          const Vec3 n = (has_minus ? 1.0 / area : -1.0 / area) * S;  // out of the owner
          const Vec3 cP = s.centre[own];
          const Vec3 d = nbr >= 0 ? s.centre[nbr] - cP : xm - cP;
          const double mksi = norm(d);
          const Vec3 ksi = (1.0 / mksi) * d;
          Vec3 skew{0, 0, 0};
          if (nbr >= 0) {
            // where the line of the centres crosses the plane of the face
            const double lam = dot(xm - cP, n) / dot(ksi, n);
            skew = (cP + lam * ksi) - xm;
          }
          const Vec3 eta = unit(v[1] - v[0]);
          m.owner[2 * f] = own + 1;
          m.owner[2 * f + 1] = nbr >= 0 ? nbr + 1 : -1;
          m.mksi[f] = mksi;
          m.area[f] = area;
          m.mvskew[f] = norm(skew);
          const Vec3 *vec[5] = {&ksi, &eta, &n, &xm, &skew};
          double *dst[5] = {m.ksi, m.eta, m.normal, m.xm, m.vskew};
          for (int q = 0; q < 5; ++q) {
            dst[q][3 * f] = vec[q]->x;
            dst[q][3 * f + 1] = vec[q]->y;
            dst[q][3 * f + 2] = vec[q]->z;
          }
          // the face in its cells' face slots: 2*ax + 1 in the minus cell, 2*ax in the plus cell
          const int32_t cells[2] = {cm, cp};
          const int slots[2] = {2 * ax + 1, 2 * ax};
          for (int q = 0; q < 2; ++q) {
            const int32_t c = cells[q];
            if (c < 0) continue;
            const size_t e = static_cast<size_t>(c) * kFaces + slots[q];
            const int32_t other = cells[q ^ 1];
            m.nelcon[e] = other >= 0 ? other + 1 : -1;
            m.cellface[e] = static_cast<int32_t>(f + 1);
            const Vec3 xmcc = xm - s.centre[c];
            m.xmcc[3 * e] = xmcc.x;
            m.xmcc[3 * e + 1] = xmcc.y;
            m.xmcc[3 * e + 2] = xmcc.z;
            m.dcca[e] = std::fabs(dot(xmcc, n));
          }
        }
  }
}

// sorted (col, face) pairs of one row
void row_entries(const System &s, int32_t r, std::vector<std::pair<int32_t, int>> &out) {
  out.clear();
  for (int f = 0; f < kFaces; ++f) {
    const int32_t col = s.nb[static_cast<size_t>(r) * kFaces + f];
    if (col >= 0) out.emplace_back(col, f);
  }
  std::sort(out.begin(), out.end());
}

}  // namespace

extern "C" {

void *sfr_sys_build(const sfr_sys_params *p) {
  if (!p || !valid(*p)) return nullptr;
  try {
    return build(*p);
  } catch (...) {
    return nullptr;
  }
}

void sfr_sys_free(void *h) { delete static_cast<System *>(h); }

int sfr_sys_info(const void *h, sfr_sys_info_t *out) {
  if (!h || !out) return -1;
  const auto &s = *static_cast<const System *>(h);
  std::memset(out, 0, sizeof(*out));
  out->neq = s.neq;
  out->nnz_full = s.nnz_full;
  out->nnz_lower = s.nnz_lower;
  out->width = kFaces;
  out->nrhs = s.p.nrhs;
  out->unsym = s.unsym ? 1 : 0;
  out->bandwidth = s.bandwidth;
  out->velocity_scale = s.velocity_scale;
  return 0;
}

int sfr_sys_csrd_full(const void *h, int32_t *ia, int32_t *ja, double *al, double *ad) {
  if (!h || !ia || !ja || !al || !ad) return -1;
  const auto &s = *static_cast<const System *>(h);
  std::vector<std::pair<int32_t, int>> e;
  int32_t k = 0;
  ia[0] = 0;
  for (int32_t r = 0; r < s.neq; ++r) {
    row_entries(s, r, e);
    for (auto &cf : e) {
      ja[k] = cf.first;
      al[k] = s.off[static_cast<size_t>(r) * kFaces + cf.second];
      ++k;
    }
    ia[r + 1] = k;
    ad[r] = s.diag[r];
  }
  return 0;
}

int sfr_sys_csrd_lower(const void *h, int32_t *ia, int32_t *ja, double *al) {
  if (!h || !ia || !ja || !al) return -1;
  const auto &s = *static_cast<const System *>(h);
  std::vector<std::pair<int32_t, int>> e;
  int32_t k = 0;
  ia[0] = 0;
  for (int32_t r = 0; r < s.neq; ++r) {
    row_entries(s, r, e);
    for (auto &cf : e) {
      if (cf.first >= r) break;
      ja[k] = cf.first;
      al[k] = s.off[static_cast<size_t>(r) * kFaces + cf.second];
      ++k;
    }
    ia[r + 1] = k;
  }
  return 0;
}

int sfr_sys_csrc(const void *h, int32_t *ia, int32_t *ja, double *a) {
  if (!h || !ia || !ja || !a) return -1;
  const auto &s = *static_cast<const System *>(h);
  std::vector<std::pair<int32_t, int>> e;
  int32_t k = 0;
  ia[0] = 0;
  double *au = a + s.nnz_lower;
  for (int32_t r = 0; r < s.neq; ++r) {
    row_entries(s, r, e);
    for (auto &cf : e) {
      if (cf.first >= r) break;
      ja[k] = cf.first;
      a[k] = s.off[static_cast<size_t>(r) * kFaces + cf.second];
      // A(col, r): the opposite face of the shared face, in col's row
      au[k] = s.off[static_cast<size_t>(cf.first) * kFaces + (cf.second ^ 1)];
      ++k;
    }
    ia[r + 1] = k;
  }
  return 0;
}

int sfr_sys_ell(const void *h, int32_t *ja, double *a) {
  if (!h || !ja || !a) return -1;
  const auto &s = *static_cast<const System *>(h);
  for (int32_t r = 0; r < s.neq; ++r)
    for (int f = 0; f < kFaces; ++f) {
      const size_t q = static_cast<size_t>(r) * kFaces + f;
      const int32_t col = s.nb[q];
      ja[q] = col >= 0 ? col : r;
      a[q] = col >= 0 ? s.off[q] : -0.0;
    }
  return 0;
}

int sfr_sys_rhs(const void *h, double *b) {
  if (!h || !b) return -1;
  const auto &s = *static_cast<const System *>(h);
  std::copy(s.rhs.begin(), s.rhs.end(), b);
  return 0;
}

int sfr_sys_numbering(const void *h, int32_t *eq_of_cell) {
  if (!h || !eq_of_cell) return -1;
  const auto &s = *static_cast<const System *>(h);
  std::copy(s.eq_of_cell.begin(), s.eq_of_cell.end(), eq_of_cell);
  return 0;
}

int sfr_sys_mesh_sizes(const void *h, int32_t *numel, int64_t *nface) {
  if (!h || !numel || !nface) return -1;
  const auto &s = *static_cast<const System *>(h);
  *numel = s.neq;
  *nface = face_count(s.p);
  return 0;
}

int sfr_sys_mesh(const void *h, const sfr_sys_mesh_t *m) {
  if (!h || !m) return -1;
  const void *need[] = {m->nelcon, m->nviz, m->cellface, m->volume, m->dcca, m->xmcc,
                        m->cdiff, m->id, m->owner, m->mksi, m->ksi, m->eta, m->area,
                        m->normal, m->xm, m->mvskew, m->vskew};
  for (const void *q : need)
    if (!q) return -1;
  try {
    export_mesh(*static_cast<const System *>(h), *m);
  } catch (...) {
    return -1;
  }
  return 0;
}

int sfr_sys_batch_params(int32_t count, int32_t nmin, int32_t nmax, uint64_t seed,
                         sfr_sys_params *out) {
  if (count < 0 || nmin < 1 || nmax < nmin || !out) return -1;
  Rng rng(seed ^ 0x510E527FADE682D1ULL);
  const double lo = std::log(static_cast<double>(nmin)), hi = std::log(static_cast<double>(nmax));
  uint64_t st = seed;
  for (int32_t b = 0; b < count; ++b) {
    sfr_sys_params p{};
    p.kind = SFR_SYS_DIFFUSION;
    int n[3];
    for (int &v : n) {
      v = static_cast<int>(std::lround(std::exp(rng.uniform(lo, hi))));
      v = std::min(std::max(v, nmin), nmax);
    }
    p.nx = n[0];
    p.ny = n[1];
    p.nz = n[2];
    double h[3] = {1.0, 1.0, 1.0};
    const int ax = static_cast<int>(rng.below(3));
    h[ax] = rng.uniform(1.0, 10.0);
    p.lx = n[0] * h[0];
    p.ly = n[1] * h[1];
    p.lz = n[2] * h[2];
    p.jitter = 0.0;
    p.log10k_lo = p.log10k_hi = rng.uniform(-1.0, 1.0);
    p.dirichlet_faces = 1 << static_cast<int>(rng.below(6));
    p.permute = 0;
    p.rcm = 1;
    p.nrhs = 1;
    p.rhs_normal = 0;
    p.seed = splitmix64(st);
    out[b] = p;
  }
  return 0;
}

}  // extern "C"
