// Airfoil C-mesh generator: a C++ restatement of the reference's MATLAB mesh
// script airfoil/naca0012.m (new-style output, naca0012.m:203-351), plus the
// new_grid.dat reader of airfoil/airfoil.cpp:80-129 and a seeded renumbering.
//
// Host-only code; it produces the input of the parallel loops, not results.

#include "op2b_mesh.h"

#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <sys/stat.h>
#include <vector>

namespace {

// linspace(a, b, n) with exact end points (MATLAB semantics).
std::vector<double> linspace(double a, double b, int n) {
  std::vector<double> v(n);
  for (int k = 0; k < n; k++) v[k] = a + k * ((b - a) / (n - 1));
  v[0] = a;
  v[n - 1] = b;
  return v;
}

// Cubic spline with not-a-knot end conditions, the default of MATLAB's
// spline(x, y, xx) when y has as many entries as x (naca0012.m:49).  Solved
// for the second derivatives M; the two end rows say that the third
// derivative is continuous at the second and second-to-last knots.
struct Spline {
  std::vector<double> x, y, M;

  Spline(const std::vector<double> &xs, const std::vector<double> &ys) : x(xs), y(ys) {
    const int n = (int)x.size();
    std::vector<double> h(n - 1);
    for (int i = 0; i < n - 1; i++) h[i] = x[i + 1] - x[i];
    // dense n x n system, solved by Gaussian elimination with partial pivoting
    std::vector<double> A((size_t)n * n, 0.0), r(n, 0.0);
    auto a = [&](int i, int j) -> double & { return A[(size_t)i * n + j]; };
    a(0, 0) = h[1];
    a(0, 1) = -(h[0] + h[1]);
    a(0, 2) = h[0];
    for (int i = 1; i < n - 1; i++) {
      a(i, i - 1) = h[i - 1];
      a(i, i) = 2.0 * (h[i - 1] + h[i]);
      a(i, i + 1) = h[i];
      r[i] = 6.0 * ((y[i + 1] - y[i]) / h[i] - (y[i] - y[i - 1]) / h[i - 1]);
    }
    a(n - 1, n - 3) = h[n - 2];
    a(n - 1, n - 2) = -(h[n - 3] + h[n - 2]);
    a(n - 1, n - 1) = h[n - 3];
    for (int k = 0; k < n; k++) {
      int p = k;
      for (int i = k + 1; i < n; i++)
        if (std::fabs(a(i, k)) > std::fabs(a(p, k))) p = i;
      if (p != k) {
        for (int j = 0; j < n; j++) std::swap(a(k, j), a(p, j));
        std::swap(r[k], r[p]);
      }
      for (int i = k + 1; i < n; i++) {
        double f = a(i, k) / a(k, k);
        if (f == 0.0) continue;
        for (int j = k; j < n; j++) a(i, j) -= f * a(k, j);
        r[i] -= f * r[k];
      }
    }
    M.assign(n, 0.0);
    for (int i = n - 1; i >= 0; i--) {
      double s = r[i];
      for (int j = i + 1; j < n; j++) s -= a(i, j) * M[j];
      M[i] = s / a(i, i);
    }
  }

  // Evaluate; points outside [x0, x_{n-1}] use the end pieces (MATLAB
  // extrapolates with the first / last polynomial).
  double operator()(double t) const {
    const int n = (int)x.size();
    int i = 0, hi = n - 2;
    if (t >= x[n - 2]) {
      i = n - 2;
    } else if (t > x[0]) {
      int lo = 0;
      while (hi - lo > 1) {
        int mid = (lo + hi) / 2;
        if (x[mid] <= t) lo = mid; else hi = mid;
      }
      i = lo;
    }
    double h = x[i + 1] - x[i];
    double a = x[i + 1] - t, b = t - x[i];
    return M[i] * a * a * a / (6.0 * h) + M[i + 1] * b * b * b / (6.0 * h) +
           (y[i] / h - M[i] * h / 6.0) * a + (y[i + 1] / h - M[i + 1] * h / 6.0) * b;
  }
};

void permute_numbering(op2b_mesh *m, uint64_t seed) {
  uint64_t st = seed;
  auto make_perm = [&](int n) {
    std::vector<int> p(n);
    for (int i = 0; i < n; i++) p[i] = i;
    for (int i = n - 1; i > 0; i--) {
      uint64_t r = op2b_splitmix64(&st);
      int j = (int)(((unsigned __int128)r * (unsigned)(i + 1)) >> 64);
      std::swap(p[i], p[j]);
    }
    return p;  // p[old] = new
  };
  // draw order: nodes, cells, edges, bedges
  std::vector<int> pn = make_perm(m->nnode), pc = make_perm(m->ncell),
                   pe = make_perm(m->nedge), pb = make_perm(m->nbedge);

  std::vector<double> x64(m->x64, m->x64 + 2 * (size_t)m->nnode);
  std::vector<float> x32(m->x32, m->x32 + 2 * (size_t)m->nnode);
  for (int n = 0; n < m->nnode; n++)
    for (int d = 0; d < 2; d++) {
      m->x64[2 * (size_t)pn[n] + d] = x64[2 * (size_t)n + d];
      m->x32[2 * (size_t)pn[n] + d] = x32[2 * (size_t)n + d];
    }
  std::vector<int> cell(m->cell, m->cell + 4 * (size_t)m->ncell);
  for (int c = 0; c < m->ncell; c++)
    for (int d = 0; d < 4; d++) m->cell[4 * (size_t)pc[c] + d] = pn[cell[4 * (size_t)c + d]];
  std::vector<int> edge(m->edge, m->edge + 2 * (size_t)m->nedge),
      ecell(m->ecell, m->ecell + 2 * (size_t)m->nedge);
  for (int e = 0; e < m->nedge; e++)
    for (int d = 0; d < 2; d++) {
      m->edge[2 * (size_t)pe[e] + d] = pn[edge[2 * (size_t)e + d]];
      m->ecell[2 * (size_t)pe[e] + d] = pc[ecell[2 * (size_t)e + d]];
    }
  std::vector<int> bedge(m->bedge, m->bedge + 2 * (size_t)m->nbedge),
      becell(m->becell, m->becell + m->nbedge), bound(m->bound, m->bound + m->nbedge);
  for (int b = 0; b < m->nbedge; b++) {
    for (int d = 0; d < 2; d++) m->bedge[2 * (size_t)pb[b] + d] = pn[bedge[2 * (size_t)b + d]];
    m->becell[pb[b]] = pc[becell[b]];
    m->bound[pb[b]] = bound[b];
  }
}

bool alloc_mesh(op2b_mesh *m) {
  m->cell = (int *)malloc(sizeof(int) * 4 * (size_t)m->ncell);
  m->edge = (int *)malloc(sizeof(int) * 2 * (size_t)m->nedge);
  m->ecell = (int *)malloc(sizeof(int) * 2 * (size_t)m->nedge);
  m->bedge = (int *)malloc(sizeof(int) * 2 * (size_t)m->nbedge);
  m->becell = (int *)malloc(sizeof(int) * (size_t)m->nbedge);
  m->bound = (int *)malloc(sizeof(int) * (size_t)m->nbedge);
  m->x64 = (double *)malloc(sizeof(double) * 2 * (size_t)m->nnode);
  m->x32 = (float *)malloc(sizeof(float) * 2 * (size_t)m->nnode);
  return m->cell && m->edge && m->ecell && m->bedge && m->becell && m->bound && m->x64 && m->x32;
}

}  // namespace

extern "C" uint64_t op2b_splitmix64(uint64_t *state) {
  uint64_t z = (*state += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

extern "C" void op2b_mesh_free(op2b_mesh *m) {
  if (!m) return;
  free(m->cell); free(m->edge); free(m->ecell); free(m->bedge);
  free(m->becell); free(m->bound); free(m->x64); free(m->x32);
  memset(m, 0, sizeof(*m));
}

extern "C" int op2b_mesh_naca0012(int I, int J, int scramble, uint64_t seed, op2b_mesh *m) {
  if (!m || I < 2 || J < 2 || (long long)3 * I * J > 0x3fffffff) return 1;
  memset(m, 0, sizeof(*m));

  // airfoil upper surface (naca0012.m:8-11)
  const int ns = 100;
  std::vector<double> xs = linspace(0.0, M_PI / 2, ns), ys(ns);
  for (int k = 0; k < ns; k++) {
    double s = std::sin(xs[k]);
    double x = s * s;
    xs[k] = x;
    ys[k] = 0.594689181 * (0.298222773 * std::sqrt(x) - 0.127125232 * x - 0.357907906 * x * x +
                           0.291984971 * x * x * x - 0.105174696 * x * x * x * x);
  }
  ys[ns - 1] = 0.0;

  // complex square-root transform and reflection (naca0012.m:17-29)
  const double x0 = 0.0077;
  std::vector<std::complex<double>> z(ns);
  for (int k = 0; k < ns; k++) z[k] = std::sqrt(std::complex<double>(xs[k], ys[k]) - x0);
  std::vector<double> sx, sy;
  for (int k = ns - 1; k >= 0; k--) {  // -conj(fliplr(z))
    sx.push_back(-z[k].real());
    sy.push_back(z[k].imag());
  }
  for (int k = 1; k < ns; k++) {  // z(2:end)
    sx.push_back(z[k].real());
    sy.push_back(z[k].imag());
  }
  Spline sp(sx, sy);

  // grid in the square-root plane (naca0012.m:45-56); MATLAB's 1-based
  // I+2..2I is 0-based I+1..2I-1
  const int ni = 3 * I + 1, nj = J + 1;
  std::vector<double> xb = linspace(-3.0, 3.0, ni), yb(ni, 0.0);
  for (int i = I + 1; i <= 2 * I - 1; i++) yb[i] = sp(xb[i]);

  m->nnode = ni * nj;
  m->ncell = 3 * I * J;
  m->nedge = (3 * I - 1) * J + 3 * I * (J - 1) + I;
  m->nbedge = I + 3 * I + 2 * J;
  if (!alloc_mesh(m)) { op2b_mesh_free(m); return 2; }

  auto node = [&](int i, int j) { return i + j * ni; };
  auto cellid = [&](int i, int j) { return i + j * 3 * I; };

  // nodes: z^2 back to the physical plane (naca0012.m:60-61), then the
  // "%f" text round trip of naca0012.m:334 / airfoil.cpp:146
  char buf[64];
  for (int i = 0; i < ni; i++) {
    std::vector<double> yg = linspace(yb[i], 3.0, nj);
    for (int j = 0; j < nj; j++) {
      double a = xb[i], b = yg[j];
      double px = a * a - b * b, py = a * b + b * a;
      int k = node(i, j);
      double v[2] = {px, py};
      for (int d = 0; d < 2; d++) {
        snprintf(buf, sizeof buf, "%f", v[d]);
        m->x64[2 * (size_t)k + d] = strtod(buf, nullptr);
        m->x32[2 * (size_t)k + d] = strtof(buf, nullptr);
      }
    }
  }

  // cells (naca0012.m:237-246)
  for (int j = 0; j < J; j++)
    for (int i = 0; i < 3 * I; i++) {
      size_t k = (size_t)cellid(i, j);
      m->cell[4 * k + 0] = node(i, j);
      m->cell[4 * k + 1] = node(i + 1, j);
      m->cell[4 * k + 2] = node(i + 1, j + 1);
      m->cell[4 * k + 3] = node(i, j + 1);
    }

  // interior edges: cut line, up, right (naca0012.m:253-281)
  size_t ie = 0;
  for (int j = 0; j < J; j++)
    for (int i = 0; i < 3 * I; i++) {
      if (j == 0 && i < I) {
        m->edge[2 * ie] = node(i, j);      m->edge[2 * ie + 1] = node(i + 1, j);
        m->ecell[2 * ie] = cellid(3 * I - 1 - i, j); m->ecell[2 * ie + 1] = cellid(i, j);
        ie++;
      }
      if (j < J - 1) {
        m->edge[2 * ie] = node(i, j + 1);  m->edge[2 * ie + 1] = node(i + 1, j + 1);
        m->ecell[2 * ie] = cellid(i, j);   m->ecell[2 * ie + 1] = cellid(i, j + 1);
        ie++;
      }
      if (i < 3 * I - 1) {
        m->edge[2 * ie] = node(i + 1, j);  m->edge[2 * ie + 1] = node(i + 1, j + 1);
        m->ecell[2 * ie] = cellid(i + 1, j); m->ecell[2 * ie + 1] = cellid(i, j);
        ie++;
      }
    }
  if ((int)ie != m->nedge) { op2b_mesh_free(m); return 3; }

  // boundary edges: airfoil, right, top, left (naca0012.m:291-321)
  size_t ib = 0;
  auto bset = [&](int n1, int n2, int c, int b) {
    m->bedge[2 * ib] = n1; m->bedge[2 * ib + 1] = n2;
    m->becell[ib] = c;     m->bound[ib] = b;
    ib++;
  };
  for (int i = I; i <= 2 * I - 1; i++) bset(node(i + 1, 0), node(i, 0), cellid(i, 0), 1);
  for (int j = 0; j < J; j++) bset(node(3 * I, j + 1), node(3 * I, j), cellid(3 * I - 1, j), 2);
  for (int i = 3 * I - 1; i >= 0; i--) bset(node(i, J), node(i + 1, J), cellid(i, J - 1), 2);
  for (int j = J - 1; j >= 0; j--) bset(node(0, j), node(0, j + 1), cellid(0, j), 2);
  if ((int)ib != m->nbedge) { op2b_mesh_free(m); return 3; }

  if (scramble) permute_numbering(m, seed);
  return 0;
}

extern "C" int op2b_mesh_write(const op2b_mesh *m, const char *path) {
  FILE *fp = fopen(path, "w");
  if (!fp) return 1;
  fprintf(fp, " %d %d %d %d \n", m->nnode, m->ncell, m->nedge, m->nbedge);
  char a[64], b[64];
  for (int n = 0; n < m->nnode; n++) {
    // x64 already holds the parsed "%f" value, so printing it again with
    // "%f" reproduces the original text
    snprintf(a, sizeof a, "%f", m->x64[2 * (size_t)n]);
    snprintf(b, sizeof b, "%f", m->x64[2 * (size_t)n + 1]);
    fprintf(fp, " %s %s \n", a, b);
  }
  for (int n = 0; n < m->ncell; n++)
    fprintf(fp, " %d %d %d %d \n", m->cell[4 * (size_t)n], m->cell[4 * (size_t)n + 1],
            m->cell[4 * (size_t)n + 2], m->cell[4 * (size_t)n + 3]);
  for (int n = 0; n < m->nedge; n++)
    fprintf(fp, " %d %d %d %d \n", m->edge[2 * (size_t)n], m->edge[2 * (size_t)n + 1],
            m->ecell[2 * (size_t)n], m->ecell[2 * (size_t)n + 1]);
  for (int n = 0; n < m->nbedge; n++)
    fprintf(fp, " %d %d %d %d \n", m->bedge[2 * (size_t)n], m->bedge[2 * (size_t)n + 1],
            m->becell[n], m->bound[n]);
  return fclose(fp) == 0 ? 0 : 2;
}

// Text input, fast path: the whole file in memory, integers parsed by hand,
// coordinates by strtod / strtof on the same tokens (so values equal the
// reference reader's, airfoil/airfoil.cpp:80-129).  Returns -1 when the text
// does not have the expected shape, so the caller can fall back to fscanf.
namespace {

bool slurp(const char *path, std::vector<char> &buf) {
  FILE *fp = fopen(path, "rb");
  if (!fp) return false;
  fseek(fp, 0, SEEK_END);
  long n = ftell(fp);
  fseek(fp, 0, SEEK_SET);
  if (n < 0) { fclose(fp); return false; }
  buf.resize((size_t)n + 1);
  size_t got = fread(buf.data(), 1, (size_t)n, fp);
  fclose(fp);
  buf[got] = 0;
  buf.resize(got + 1);
  return true;
}

struct Cursor {
  const char *p, *end;
  void skip() { while (p < end && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) p++; }
  bool integer(int &v) {
    skip();
    bool neg = false;
    if (p < end && (*p == '-' || *p == '+')) neg = *p++ == '-';
    if (p >= end || *p < '0' || *p > '9') return false;
    long long x = 0;
    while (p < end && *p >= '0' && *p <= '9') {
      x = x * 10 + (*p++ - '0');
      if (x > 2147483648LL) return false;
    }
    if (p < end && *p != ' ' && *p != '\n' && *p != '\r' && *p != '\t') return false;
    v = (int)(neg ? -x : x);
    return true;
  }
  bool real(double &d, float &f) {
    skip();
    const char *t = p;
    while (p < end && *p != ' ' && *p != '\n' && *p != '\r' && *p != '\t') p++;
    if (p == t || p - t > 127) return false;
    char tok[128];
    memcpy(tok, t, p - t);
    tok[p - t] = 0;
    char *e1, *e2;
    d = strtod(tok, &e1);
    f = strtof(tok, &e2);
    return *e1 == 0 && *e2 == 0;
  }
};

int parse_text(const char *path, op2b_mesh *m) {
  std::vector<char> buf;
  if (!slurp(path, buf)) return 1;
  Cursor c{buf.data(), buf.data() + buf.size() - 1};
  if (!c.integer(m->nnode) || !c.integer(m->ncell) || !c.integer(m->nedge) ||
      !c.integer(m->nbedge) || m->nnode <= 0 || m->ncell <= 0 || m->nedge <= 0 ||
      m->nbedge <= 0)
    return -1;
  if (!alloc_mesh(m)) return 3;
  for (int n = 0; n < m->nnode; n++)
    for (int k = 0; k < 2; k++)
      if (!c.real(m->x64[2 * (size_t)n + k], m->x32[2 * (size_t)n + k])) return -1;
  for (size_t i = 0; i < 4 * (size_t)m->ncell; i++)
    if (!c.integer(m->cell[i])) return -1;
  for (int n = 0; n < m->nedge; n++)
    if (!c.integer(m->edge[2 * (size_t)n]) || !c.integer(m->edge[2 * (size_t)n + 1]) ||
        !c.integer(m->ecell[2 * (size_t)n]) || !c.integer(m->ecell[2 * (size_t)n + 1]))
      return -1;
  for (int n = 0; n < m->nbedge; n++)
    if (!c.integer(m->bedge[2 * (size_t)n]) || !c.integer(m->bedge[2 * (size_t)n + 1]) ||
        !c.integer(m->becell[n]) || !c.integer(m->bound[n]))
      return -1;
  return 0;
}

}  // namespace

extern "C" int op2b_mesh_read(const char *path, op2b_mesh *m) {
  memset(m, 0, sizeof(*m));
  const int fast = parse_text(path, m);
  if (fast >= 0) {
    if (fast) op2b_mesh_free(m);
    return fast;
  }
  op2b_mesh_free(m);  // unexpected layout: the reference's own scanf reading
  memset(m, 0, sizeof(*m));
  FILE *fp = fopen(path, "r");
  if (!fp) return 1;
  int rc = 0;
  if (fscanf(fp, "%d %d %d %d \n", &m->nnode, &m->ncell, &m->nedge, &m->nbedge) != 4 ||
      m->nnode <= 0 || m->ncell <= 0 || m->nedge <= 0 || m->nbedge <= 0) {
    fclose(fp);
    return 2;
  }
  if (!alloc_mesh(m)) { fclose(fp); op2b_mesh_free(m); return 3; }
  char a[128], b[128];
  for (int n = 0; n < m->nnode && !rc; n++) {
    if (fscanf(fp, "%127s %127s \n", a, b) != 2) { rc = 2; break; }
    m->x64[2 * (size_t)n] = strtod(a, nullptr);
    m->x64[2 * (size_t)n + 1] = strtod(b, nullptr);
    m->x32[2 * (size_t)n] = strtof(a, nullptr);
    m->x32[2 * (size_t)n + 1] = strtof(b, nullptr);
  }
  for (int n = 0; n < m->ncell && !rc; n++)
    if (fscanf(fp, "%d %d %d %d \n", &m->cell[4 * (size_t)n], &m->cell[4 * (size_t)n + 1],
               &m->cell[4 * (size_t)n + 2], &m->cell[4 * (size_t)n + 3]) != 4) rc = 2;
  for (int n = 0; n < m->nedge && !rc; n++)
    if (fscanf(fp, "%d %d %d %d \n", &m->edge[2 * (size_t)n], &m->edge[2 * (size_t)n + 1],
               &m->ecell[2 * (size_t)n], &m->ecell[2 * (size_t)n + 1]) != 4) rc = 2;
  for (int n = 0; n < m->nbedge && !rc; n++)
    if (fscanf(fp, "%d %d %d %d \n", &m->bedge[2 * (size_t)n], &m->bedge[2 * (size_t)n + 1],
               &m->becell[n], &m->bound[n]) != 4) rc = 2;
  fclose(fp);
  if (rc) op2b_mesh_free(m);
  return rc;
}

// ------------------------------------------------------ binary mesh cache --
// "OP2BMSH1" header, the four sizes, the size and modification time of the
// text file it was made from, an FNV-1a hash of the payload, then the arrays
// (cell, edge, ecell, bedge, becell, bound, x64, x32) in host byte order.

namespace {

struct BinHeader {
  char magic[8];
  int32_t version, nnode, ncell, nedge, nbedge, pad;
  int64_t src_size, src_mtime_ns;
  uint64_t hash;
};

struct Part {
  void *p;
  size_t bytes;
};

std::vector<Part> parts(const op2b_mesh *m) {
  return {{m->cell, sizeof(int) * 4 * (size_t)m->ncell},
          {m->edge, sizeof(int) * 2 * (size_t)m->nedge},
          {m->ecell, sizeof(int) * 2 * (size_t)m->nedge},
          {m->bedge, sizeof(int) * 2 * (size_t)m->nbedge},
          {m->becell, sizeof(int) * (size_t)m->nbedge},
          {m->bound, sizeof(int) * (size_t)m->nbedge},
          {m->x64, sizeof(double) * 2 * (size_t)m->nnode},
          {m->x32, sizeof(float) * 2 * (size_t)m->nnode}};
}

// FNV-1a over 8-byte words (then the tail bytes)
uint64_t fnv1a(const std::vector<Part> &ps) {
  uint64_t h = 0xcbf29ce484222325ull;
  for (const Part &q : ps) {
    const unsigned char *b = (const unsigned char *)q.p;
    size_t i = 0;
    for (; i + 8 <= q.bytes; i += 8) {
      uint64_t w;
      memcpy(&w, b + i, 8);
      h = (h ^ w) * 0x100000001b3ull;
    }
    for (; i < q.bytes; i++) h = (h ^ b[i]) * 0x100000001b3ull;
  }
  return h;
}

bool file_stamp(const char *path, int64_t &size, int64_t &mtime_ns) {
  struct stat st;
  if (!path || stat(path, &st) != 0) return false;
  size = (int64_t)st.st_size;
  mtime_ns = (int64_t)st.st_mtim.tv_sec * 1000000000LL + st.st_mtim.tv_nsec;
  return true;
}

int write_bin(const op2b_mesh *m, const char *path, int64_t src_size, int64_t src_mtime) {
  BinHeader h;
  memset(&h, 0, sizeof h);
  memcpy(h.magic, "OP2BMSH1", 8);
  h.version = 1;
  h.nnode = m->nnode; h.ncell = m->ncell; h.nedge = m->nedge; h.nbedge = m->nbedge;
  h.src_size = src_size;
  h.src_mtime_ns = src_mtime;
  std::vector<Part> ps = parts(m);
  h.hash = fnv1a(ps);
  std::string tmp = std::string(path) + ".tmp";
  FILE *fp = fopen(tmp.c_str(), "wb");
  if (!fp) return 1;
  bool ok = fwrite(&h, sizeof h, 1, fp) == 1;
  for (const Part &q : ps) ok = ok && fwrite(q.p, 1, q.bytes, fp) == q.bytes;
  ok = (fclose(fp) == 0) && ok;
  if (!ok || rename(tmp.c_str(), path) != 0) {
    remove(tmp.c_str());
    return 2;
  }
  return 0;
}

// 0 ok; 1 missing; 2 bad or stale (want_size >= 0: must match the stamp)
int read_bin(const char *path, op2b_mesh *m, int64_t want_size, int64_t want_mtime) {
  memset(m, 0, sizeof(*m));
  FILE *fp = fopen(path, "rb");
  if (!fp) return 1;
  BinHeader h;
  if (fread(&h, sizeof h, 1, fp) != 1 || memcmp(h.magic, "OP2BMSH1", 8) != 0 || h.version != 1 ||
      h.nnode <= 0 || h.ncell <= 0 || h.nedge <= 0 || h.nbedge <= 0 ||
      (want_size >= 0 && (h.src_size != want_size || h.src_mtime_ns != want_mtime))) {
    fclose(fp);
    return 2;
  }
  m->nnode = h.nnode; m->ncell = h.ncell; m->nedge = h.nedge; m->nbedge = h.nbedge;
  if (!alloc_mesh(m)) {
    fclose(fp);
    op2b_mesh_free(m);
    return 3;
  }
  std::vector<Part> ps = parts(m);
  bool ok = true;
  for (const Part &q : ps) ok = ok && fread(q.p, 1, q.bytes, fp) == q.bytes;
  fclose(fp);
  if (!ok || fnv1a(ps) != h.hash) {
    op2b_mesh_free(m);
    return 2;
  }
  return 0;
}

}  // namespace

extern "C" int op2b_mesh_write_bin(const op2b_mesh *m, const char *path) {
  return write_bin(m, path, -1, -1);
}

extern "C" int op2b_mesh_read_bin(const char *path, op2b_mesh *out) {
  return read_bin(path, out, -1, -1);
}

extern "C" int op2b_mesh_read_cached(const char *text_path, const char *cache_path,
                                     op2b_mesh *out) {
  int64_t size = 0, mtime = 0;
  if (!file_stamp(text_path, size, mtime)) return 1;
  if (cache_path && read_bin(cache_path, out, size, mtime) == 0) return 0;
  int rc = op2b_mesh_read(text_path, out);
  if (rc == 0 && cache_path) write_bin(out, cache_path, size, mtime);  // best effort
  return rc;
}

// ------------------------------------------------------------ jac1 / jac2 --

extern "C" int op2b_jac_sizes(int NN, int *nnode, int *nedge) {
  if (NN < 3) return 1;
  *nnode = (NN - 1) * (NN - 1);
  *nedge = (NN - 1) * (NN - 1) + 4 * (NN - 1) * (NN - 2);
  return 0;
}

// jac1/jac.cpp:82-117 and jac2/jac.cpp:68-108; A and r strides differ
template <class AT>
static int jac_mesh(int NN, int *pp, AT *A, int astride, float *r, int rstride) {
  int nnode, nedge;
  if (op2b_jac_sizes(NN, &nnode, &nedge)) return -1;
  for (int k = 0; k < astride * nedge; k++) A[k] = 0;
  for (int k = 0; k < rstride * nnode; k++) r[k] = 0.0f;
  int e = 0;
  for (int i = 1; i < NN; i++)
    for (int j = 1; j < NN; j++) {
      int n = i - 1 + (j - 1) * (NN - 1);
      pp[2 * e] = n;
      pp[2 * e + 1] = n;
      A[astride * e] = (AT)-1.0f;
      e++;
      for (int pass = 0; pass < 4; pass++) {
        int i2 = i, j2 = j;
        if (pass == 0) i2 += -1;
        if (pass == 1) i2 += 1;
        if (pass == 2) j2 += -1;
        if (pass == 3) j2 += 1;
        if (i2 == 0 || i2 == NN || j2 == 0 || j2 == NN) {
          r[rstride * n] += 0.25f;
        } else {
          pp[2 * e] = n;
          pp[2 * e + 1] = i2 - 1 + (j2 - 1) * (NN - 1);
          A[astride * e] = (AT)0.25f;
          e++;
        }
      }
    }
  return e == nedge ? nedge : -1;
}

extern "C" int op2b_mesh_jac1(int NN, int *pp, float *A, float *r) {
  return jac_mesh<float>(NN, pp, A, 1, r, 1);
}

extern "C" int op2b_mesh_jac2(int NN, int *pp, double *A, float *r) {
  return jac_mesh<double>(NN, pp, A, 3, r, 2);
}
