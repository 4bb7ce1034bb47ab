// Symmetric eigen-decomposition for kmer2pca.  The reference hands the
// covariance matrix to LAPACK dsyev (kmer2pca.c:107-138), prints every
// eigenvalue in ascending order (kmer2pca.c:245-253) and projects the samples
// onto the eigenvectors of the `dimensions` largest ones (kmer2pca.c:141-168),
// so only those few vectors are computed here.  Host code: the matrix is
// n_features x n_features (1,024 for 5-mers); its O(nf^3) reduction takes a
// fraction of a second on the host threads, while the O(n_samples nf^2)
// covariance and the projections run on the GPU.
//
// Method (Golub and Van Loan, Matrix Computations, 4th ed., 8.3.1, 8.4.1 and
// 8.2.2; written for this library):
//  1. Householder reduction Q^T C Q = T to tridiagonal form, one reflector per
//     column.  Each step's rank-2 update of the trailing block and the next
//     step's matrix-vector product share one pass over the block's rows.
//  2. Every eigenvalue of T by bisection on Sturm counts, the brackets of the
//     other eigenvalues tightened by every count.
//  3. The vectors of the wanted eigenvalues by inverse iteration on T (LU with
//     partial pivoting of T - lambda I), re-orthogonalised against the wanted
//     vectors of the same cluster.
//  4. Back-transformation v = Q y with the stored reflectors.
// Eigenvectors are defined up to sign; each one is returned with its
// largest-magnitude entry (the first one, on ties) positive.
#include <algorithm>
#include <atomic>
#include <cfloat>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <functional>
#include <mutex>
#include <thread>
#include <vector>

#include "host_internal.h"

namespace {

// Fork-join over row ranges on persistent host threads (the caller takes the
// first range).  One run() per tridiagonalisation step.
class RowPool {
 public:
  explicit RowPool(int threads) : n_(std::max(1, threads)) {
    for (int w = 1; w < n_; ++w) th_.emplace_back([this, w]() { worker(w); });
  }
  ~RowPool() {
    {
      std::lock_guard<std::mutex> g(m_);
      stop_ = true;
      ++gen_;
    }
    cv_.notify_all();
    for (auto& t : th_) t.join();
  }
  int size() const { return n_; }
  // f(lo, hi) over [begin, end) cut into size() ranges.
  void run(int64_t begin, int64_t end, const std::function<void(int64_t, int64_t)>& f) {
    if (n_ == 1 || end - begin < 2) {
      if (end > begin) f(begin, end);
      return;
    }
    {
      std::lock_guard<std::mutex> g(m_);
      f_ = &f;
      begin_ = begin;
      end_ = end;
      pending_ = n_ - 1;
      ++gen_;
    }
    cv_.notify_all();
    range(0, f);
    std::unique_lock<std::mutex> g(m_);
    done_.wait(g, [this]() { return pending_ == 0; });
    f_ = nullptr;
  }

 private:
  void range(int w, const std::function<void(int64_t, int64_t)>& f) {
    const int64_t len = end_ - begin_;
    const int64_t lo = begin_ + len * w / n_, hi = begin_ + len * (w + 1) / n_;
    if (hi > lo) f(lo, hi);
  }
  void worker(int w) {
    uint64_t seen = 0;
    for (;;) {
      const std::function<void(int64_t, int64_t)>* f;
      {
        std::unique_lock<std::mutex> g(m_);
        cv_.wait(g, [&]() { return gen_ != seen; });
        seen = gen_;
        if (stop_) return;
        f = f_;
      }
      range(w, *f);
      std::lock_guard<std::mutex> g(m_);
      if (--pending_ == 0) done_.notify_one();
    }
  }
  int n_;
  std::vector<std::thread> th_;
  std::mutex m_;
  std::condition_variable cv_, done_;
  const std::function<void(int64_t, int64_t)>* f_ = nullptr;
  int64_t begin_ = 0, end_ = 0;
  int pending_ = 0;
  uint64_t gen_ = 0;
  bool stop_ = false;
};

int host_threads() { return (int)std::min(16u, std::max(1u, std::thread::hardware_concurrency())); }

// Reflector H = I - tau u u^T (u[0] = 1) with H x = beta e_1, x of length L.
// u[1..L-1] is written; returns tau (0 when x[1..] is zero: H = I, beta = x[0]).
double householder(const double* x, int64_t L, double* u, double* beta) {
  const double alpha = x[0];
  double sigma = 0;
  for (int64_t i = 1; i < L; ++i) sigma += x[i] * x[i];
  u[0] = 1.0;
  if (sigma == 0.0) {
    for (int64_t i = 1; i < L; ++i) u[i] = 0.0;
    *beta = alpha;
    return 0.0;
  }
  const double norm = std::sqrt(alpha * alpha + sigma);
  const double b = alpha <= 0 ? norm : -norm;
  const double scale = 1.0 / (alpha - b);
  for (int64_t i = 1; i < L; ++i) u[i] = x[i] * scale;
  *beta = b;
  return (b - alpha) / b;
}

// Tridiagonal T (diagonal d[0..n-1], off-diagonal e[0..n-2]) of the n x n
// symmetric A (row-major, overwritten).  Reflector k (k = 0 .. n-3) acts on
// indices k+1 .. n-1: u_k is stored in A[k][k+1 ..] and tau_k in tau[k].
void tridiagonalize(double* A, int64_t n, double* d, double* e, double* tau, RowPool& pool) {
  if (n == 1) {
    d[0] = A[0];
    return;
  }
  std::vector<double> u(n), p(n), w(n), un(n), pn(n);
  double beta = 0, tk = 0;
  auto row = [&](int64_t r) { return A + r * n; };
  if (n >= 3) {
    tk = householder(row(0) + 1, n - 1, u.data(), &beta);
    // p = tau A22 u over rows 1 .. n-1
    pool.run(1, n, [&](int64_t lo, int64_t hi) {
      for (int64_t g = lo; g < hi; ++g) {
        const double* a = row(g) + 1;
        double s = 0;
        for (int64_t j = 0; j < n - 1; ++j) s += a[j] * u[j];
        p[g - 1] = tk * s;
      }
    });
  }
  for (int64_t k = 0; k + 2 < n; ++k) {
    const int64_t m = n - k - 1;  // trailing block: indices k+1 .. n-1
    d[k] = row(k)[k];
    e[k] = beta;
    tau[k] = tk;
    std::memcpy(row(k) + k + 1, u.data(), sizeof(double) * m);
    if (tk != 0.0) {
      double pu = 0;
      for (int64_t j = 0; j < m; ++j) pu += p[j] * u[j];
      const double K = 0.5 * tk * pu;
      for (int64_t j = 0; j < m; ++j) w[j] = p[j] - K * u[j];
      double* a = row(k + 1) + k + 1;  // the next pivot row, whole
      for (int64_t j = 0; j < m; ++j) a[j] -= u[0] * w[j] + w[0] * u[j];
    }
    const bool next = k + 3 < n;
    double bn = 0, tn = 0;
    if (next) tn = householder(row(k + 1) + k + 2, m - 1, un.data(), &bn);
    // rows k+2 .. n-1: this step's update, then the next step's product
    auto pass = [&](int64_t lo, int64_t hi) {
      for (int64_t i = lo; i < hi; ++i) {
        double* a = row(k + 1 + i) + k + 1;
        if (tk != 0.0) {
          const double ui = u[i], wi = w[i];
          for (int64_t j = 1; j < m; ++j) a[j] -= ui * w[j] + wi * u[j];
        }
        if (next) {
          double s = 0;
          for (int64_t j = 1; j < m; ++j) s += a[j] * un[j - 1];
          pn[i - 1] = tn * s;
        }
      }
    };
    if (m > 160) pool.run(1, m, pass);
    else pass(1, m);
    if (next) {
      u.swap(un);
      p.swap(pn);
      beta = bn;
      tk = tn;
    }
  }
  d[n - 2] = row(n - 2)[n - 2];
  d[n - 1] = row(n - 1)[n - 1];
  e[n - 2] = row(n - 2)[n - 1];
}

// Number of eigenvalues of T that are <= x (Sturm count with the pivots kept
// away from zero by pivmin).
int64_t sturm_count(const double* d, const double* e2, int64_t n, double x, double pivmin) {
  int64_t c = 0;
  double q = d[0] - x;
  if (std::fabs(q) < pivmin) q = -pivmin;
  c += q <= 0;
  for (int64_t i = 1; i < n; ++i) {
    q = d[i] - x - e2[i - 1] / q;
    if (std::fabs(q) < pivmin) q = -pivmin;
    c += q <= 0;
  }
  return c;
}

// All eigenvalues of T, ascending.  Eigenvalue j is the point where the count
// passes from j to j+1; each thread bisects a contiguous run of indices and
// every count it takes tightens the brackets of the whole run.
void eigenvalues_bisect(const double* d, const double* e, int64_t n, double* lam, RowPool& pool) {
  std::vector<double> e2(std::max<int64_t>(n - 1, 1));
  double lo = d[0], hi = d[0], emax2 = 0;
  for (int64_t i = 0; i < n; ++i) {
    const double r = (i > 0 ? std::fabs(e[i - 1]) : 0) + (i + 1 < n ? std::fabs(e[i]) : 0);
    lo = std::min(lo, d[i] - r);
    hi = std::max(hi, d[i] + r);
    if (i + 1 < n) {
      e2[i] = e[i] * e[i];
      emax2 = std::max(emax2, e2[i]);
    }
  }
  const double tnorm = std::max(std::fabs(lo), std::fabs(hi));
  const double pivmin = DBL_MIN * std::max(1.0, emax2);
  const double pad = 2 * DBL_EPSILON * tnorm + 2 * pivmin;
  lo -= pad;
  hi += pad;
  pool.run(0, n, [&](int64_t a, int64_t b) {
    std::vector<double> L(b - a, lo), U(b - a, hi);
    for (int64_t j = a; j < b; ++j) {
      double l = L[j - a], u = U[j - a];
      for (int it = 0; it < 200; ++it) {
        const double tol = 2 * DBL_EPSILON * std::max(std::fabs(l), std::fabs(u)) + DBL_EPSILON * tnorm + pivmin;
        const double mid = l + 0.5 * (u - l);
        if (u - l <= tol || mid <= l || mid >= u) break;
        const int64_t c = sturm_count(d, e2.data(), n, mid, pivmin);
        // eigenvalues with index < c are <= mid, the others above it
        for (int64_t q = std::max(a, j); q < b; ++q) {
          if (q < c) U[q - a] = std::min(U[q - a], mid);
          else L[q - a] = std::max(L[q - a], mid);
        }
        l = L[j - a];
        u = U[j - a];
      }
      lam[j] = l + 0.5 * (u - l);
    }
  });
}

// Inverse iteration on T for eigenvalue lam: y with T y ~ lam y, ||y|| = 1,
// orthogonal to the vectors in `others`.
void inverse_iteration(const double* d, const double* e, int64_t n, double lam, double tnorm,
                       const std::vector<const double*>& others, uint64_t seed, double* y) {
  std::vector<double> dl(n), dd(n), du(n), du2(n), b(n);
  std::vector<unsigned char> swapped(n, 0);
  for (int64_t i = 0; i < n; ++i) {
    dd[i] = d[i] - lam;
    if (i + 1 < n) dl[i] = du[i] = e[i];
    du2[i] = 0;
  }
  const double tiny = std::max(DBL_EPSILON * tnorm, DBL_MIN);
  for (int64_t i = 0; i + 1 < n; ++i) {
    if (std::fabs(dd[i]) >= std::fabs(dl[i])) {
      if (dd[i] == 0.0) dd[i] = tiny;
      const double l = dl[i] / dd[i];
      dl[i] = l;
      dd[i + 1] -= l * du[i];
    } else {
      const double l = dd[i] / dl[i];
      const double di1 = dd[i + 1], dui = du[i];
      dd[i] = dl[i];
      dl[i] = l;
      du[i] = di1;
      dd[i + 1] = dui - l * di1;
      if (i + 2 < n) {
        du2[i] = du[i + 1];
        du[i + 1] = -l * du[i + 1];
      }
      swapped[i] = 1;
    }
  }
  for (int64_t i = 0; i < n; ++i)
    if (dd[i] == 0.0) dd[i] = tiny;
  // a fixed pseudo-random start (splitmix64)
  uint64_t s = seed * 0x9E3779B97F4A7C15ull + 1;
  for (int64_t i = 0; i < n; ++i) {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    y[i] = (double)(z >> 11) * (1.0 / 9007199254740992.0) - 0.5;
  }
  auto orthonormalize = [&]() {
    for (const double* o : others) {
      double dot = 0;
      for (int64_t i = 0; i < n; ++i) dot += o[i] * y[i];
      for (int64_t i = 0; i < n; ++i) y[i] -= dot * o[i];
    }
    double nrm = 0;
    for (int64_t i = 0; i < n; ++i) nrm += y[i] * y[i];
    nrm = std::sqrt(nrm);
    if (nrm == 0.0) {
      y[s % n] = 1.0;
      nrm = 1.0;
    }
    for (int64_t i = 0; i < n; ++i) y[i] /= nrm;
  };
  orthonormalize();
  for (int it = 0; it < 4; ++it) {
    std::memcpy(b.data(), y, sizeof(double) * n);
    for (int64_t i = 0; i + 1 < n; ++i) {
      if (swapped[i]) std::swap(b[i], b[i + 1]);
      b[i + 1] -= dl[i] * b[i];
    }
    for (int64_t i = n - 1; i >= 0; --i) {
      double v = b[i];
      if (i + 1 < n) v -= du[i] * y[i + 1];
      if (i + 2 < n) v -= du2[i] * y[i + 2];
      y[i] = v / dd[i];
      if (!std::isfinite(y[i])) y[i] = 0.0;
    }
    orthonormalize();
  }
}

}  // namespace

namespace swgpu {

bool pca_eigen_diagonal(const double* A, int64_t n, int64_t n_vectors, double* eigenvalues, double* vectors) {
  for (int64_t i = 0; i < n; ++i)
    for (int64_t j = 0; j < n; ++j)
      if (j != i && A[i * n + j] != 0.0) return false;
  // A diagonal matrix (the zero matrix of fewer than four samples among
  // them) has the unit vectors as eigenvectors.  Equal eigenvalues leave the
  // basis open; this takes the one dsyev returns, whose tridiagonal QL ends
  // with a selection sort: for each position in turn the first strictly
  // smallest value of the rest is swapped in.
  std::vector<double> dv(n);
  std::vector<int64_t> id(n);
  for (int64_t i = 0; i < n; ++i) {
    dv[i] = A[i * n + i];
    id[i] = i;
  }
  for (int64_t i = 0; i + 1 < n; ++i) {
    int64_t k = i;
    for (int64_t j = i + 1; j < n; ++j)
      if (dv[j] < dv[k]) k = j;
    if (k != i) {
      std::swap(dv[i], dv[k]);
      std::swap(id[i], id[k]);
    }
  }
  std::copy(dv.begin(), dv.end(), eigenvalues);
  for (int64_t v = 0; v < n_vectors; ++v) {
    double* y = vectors + v * n;
    std::fill(y, y + n, 0.0);
    y[id[n - 1 - v]] = 1.0;
  }
  return true;
}

void pca_vectors_from_tridiagonal(const double* A, const double* tau, const double* d, const double* e, int64_t n,
                                  const double* eigenvalues, int64_t n_vectors, double* vectors) {
  if (n_vectors == 0) return;
  double tnorm = 0;
  for (int64_t i = 0; i < n; ++i)
    tnorm = std::max(tnorm, std::fabs(d[i]) + (i > 0 ? std::fabs(e[i - 1]) : 0) + (i + 1 < n ? std::fabs(e[i]) : 0));
  // wanted eigenvalues, largest first; clusters (gaps below 1e-3 ||T||) are
  // separated by a few ulps and orthogonalised against each other
  const double cluster_gap = 1e-3 * tnorm, sep = 10 * DBL_EPSILON * std::max(tnorm, DBL_MIN);
  std::vector<double> lam(n_vectors);
  for (int64_t v = 0; v < n_vectors; ++v) {
    lam[v] = eigenvalues[n - 1 - v];
    if (v > 0 && lam[v] >= lam[v - 1] - sep) lam[v] = lam[v - 1] - sep;
  }
  for (int64_t v = 0; v < n_vectors; ++v) {
    std::vector<const double*> others;
    for (int64_t o = v - 1; o >= 0 && lam[o] - lam[v] < cluster_gap; --o) others.push_back(vectors + o * n);
    double* y = vectors + v * n;
    inverse_iteration(d, e, n, lam[v], tnorm, others, (uint64_t)v + 1, y);
  }
  // back to the basis of the covariance matrix: v = H_0 H_1 ... H_{n-3} y
  RowPool pool(n >= 256 ? (int)std::min<int64_t>(host_threads(), n_vectors) : 1);
  pool.run(0, n_vectors, [&](int64_t a, int64_t b) {
    for (int64_t v = a; v < b; ++v) {
      double* y = vectors + v * n;
      for (int64_t k = n - 3; k >= 0; --k) {
        if (tau[k] == 0.0) continue;
        const double* u = A + k * n + k + 1;
        const int64_t m = n - k - 1;
        double s = 0;
        for (int64_t j = 0; j < m; ++j) s += u[j] * y[k + 1 + j];
        s *= tau[k];
        for (int64_t j = 0; j < m; ++j) y[k + 1 + j] -= s * u[j];
      }
      int64_t big = 0;
      for (int64_t i = 1; i < n; ++i)
        if (std::fabs(y[i]) > std::fabs(y[big])) big = i;
      if (y[big] < 0)
        for (int64_t i = 0; i < n; ++i) y[i] = -y[i];
    }
  });
}

}  // namespace swgpu

extern "C" swe_status swe_pca_eigen(const double* cov, int64_t n_features, int64_t n_vectors, double* eigenvalues,
                                    double* vectors) {
  const int64_t n = n_features;
  if (n < 0 || n_vectors < 0 || n_vectors > n || (n > 0 && (!cov || !eigenvalues)) ||
      (n_vectors > 0 && !vectors))
    return SWE_ERR_INVALID;
  if (n == 0) return SWE_OK;
  if ((uint64_t)n > (uint64_t)1 << 24) return SWE_ERR_INVALID;
  std::vector<double> A;
  try {
    A.assign(cov, cov + n * n);
  } catch (const std::bad_alloc&) {
    return SWE_ERR_OOM;
  }
  for (double v : A)
    if (!std::isfinite(v)) return SWE_ERR_INVALID;
  if (swgpu::pca_eigen_diagonal(A.data(), n, n_vectors, eigenvalues, vectors)) return SWE_OK;
  std::vector<double> d(n), e(std::max<int64_t>(n - 1, 1), 0.0), tau(std::max<int64_t>(n - 2, 1), 0.0);
  {
    RowPool pool(n >= 256 ? host_threads() : 1);
    tridiagonalize(A.data(), n, d.data(), e.data(), tau.data(), pool);
    eigenvalues_bisect(d.data(), e.data(), n, eigenvalues, pool);
  }
  swgpu::pca_vectors_from_tridiagonal(A.data(), tau.data(), d.data(), e.data(), n, eigenvalues, n_vectors, vectors);
  return SWE_OK;
}
