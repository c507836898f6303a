// ORACLE -- test infrastructure only: a from-scratch implementation of the
// part of the HPTT API (High-Performance Tensor Transposition, a third-party
// library TCCG depends on and that is not installed here) which TCCG's
// generated GETT code calls (tccg/gett.py:346-391, 700-753, 1298-1375):
//
//   auto plan = hptt::create_plan(perm, dim, alpha, A, sizeA, outerSizeA,
//                                 beta, B, outerSizeB, hptt::ESTIMATE, numThreads);
//   new hptt::Transpose<float>(*plan);          // per-team copy
//   plan->setInputPtr(A); plan->setOutputPtr(B);
//   plan->resetThreadIds(); plan->addThreadId(omp_get_thread_num());
//   plan->execute_expert<streamingStores, spawnThreads, betaIsZero>();
//   plan->execute();
//
// Semantics (HPTT's documentation): B[perm(i)] = alpha * A[i] + beta * B[perm(i)],
// where dimension j of B is dimension perm[j] of A; sizeA[] are A's extents,
// outerSizeA / outerSizeB the (padded) extents of the allocations (NULL =
// dense); column-major, first index stride one. With spawnThreads = false the
// calling threads cooperate: every thread registered with addThreadId calls
// execute_expert and processes its own share.
//
// Used only to compile TCCG's emitted GETT candidates into CPU checkers and
// the timed CPU baseline; the timing therefore measures TCCG's GETT with this
// transposition, not with HPTT itself.
#pragma once
#include <omp.h>

#include <algorithm>
#include <cstdint>
#include <memory>
#include <mutex>
#include <vector>

namespace hptt {

enum SelectionMethod { ESTIMATE, MEASURE, PATIENT, CRAZY };

template <typename T>
class Transpose {
 public:
  Transpose(const int* sizeA, const int* perm, const int* outerSizeA, const int* outerSizeB,
            int dim, const T* A, T alpha, T* B, T beta, int numThreads)
      : dim_(dim), A_(A), B_(B), alpha_(alpha), beta_(beta), numThreads_(numThreads) {
    std::vector<int64_t> strideA(dim), strideB(dim);
    int64_t s = 1;
    for (int i = 0; i < dim; ++i) {
      strideA[i] = s;
      s *= outerSizeA ? outerSizeA[i] : sizeA[i];
    }
    s = 1;
    for (int j = 0; j < dim; ++j) {
      strideB[j] = s;
      s *= outerSizeB ? outerSizeB[j] : sizeA[perm[j]];
    }
    total_ = 1;
    for (int j = 0; j < dim; ++j) {
      ext_.push_back(sizeA[perm[j]]);
      sa_.push_back(strideA[perm[j]]);
      sb_.push_back(strideB[j]);
      total_ *= sizeA[perm[j]];
    }
  }
  Transpose(const Transpose& o)
      : dim_(o.dim_), A_(o.A_), B_(o.B_), alpha_(o.alpha_), beta_(o.beta_),
        numThreads_(o.numThreads_), total_(o.total_), ext_(o.ext_), sa_(o.sa_), sb_(o.sb_),
        threadIds_(o.threadIds_) {}

  void setInputPtr(const T* A) { A_ = A; }
  void setOutputPtr(T* B) { B_ = B; }
  void resetThreadIds() {
    std::lock_guard<std::mutex> g(mu_);
    threadIds_.clear();
  }
  void addThreadId(int id) {
    std::lock_guard<std::mutex> g(mu_);
    threadIds_.push_back(id);
  }

  template <bool useStreamingStores, bool spawnThreads, bool betaIsZero>
  void execute_expert() {
    if (spawnThreads) {
      const int nt = std::max(1, numThreads_);
#pragma omp parallel num_threads(nt)
      run_share<betaIsZero>(omp_get_thread_num(), omp_get_num_threads());
      return;
    }
    int me = 0, n = 1;
    {
      std::lock_guard<std::mutex> g(mu_);
      std::vector<int> ids = threadIds_;
      std::sort(ids.begin(), ids.end());
      n = std::max<int>(1, (int)ids.size());
      const int tid = omp_get_thread_num();
      for (int i = 0; i < (int)ids.size(); ++i)
        if (ids[i] == tid) me = i;
    }
    run_share<betaIsZero>(me, n);
  }

  void execute() {
    if (beta_ == T(0))
      execute_expert<false, true, true>();
    else
      execute_expert<false, true, false>();
  }

 private:
  // share `part` of `parts` of the output, in B's linear (column-major) order
  template <bool betaIsZero>
  void run_share(int part, int parts) {
    const int64_t chunk = (total_ + parts - 1) / parts;
    const int64_t lo = std::min<int64_t>(total_, chunk * part);
    const int64_t hi = std::min<int64_t>(total_, lo + chunk);
    if (lo >= hi) return;
    std::vector<int64_t> idx(dim_);
    int64_t l = lo, oa = 0, ob = 0;
    for (int j = 0; j < dim_; ++j) {
      idx[j] = l % ext_[j];
      l /= ext_[j];
      oa += idx[j] * sa_[j];
      ob += idx[j] * sb_[j];
    }
    const int64_t n0 = ext_[0], sa0 = sa_[0];
    for (int64_t i = lo; i < hi;) {
      // inner run along output dim 0 (stride one in B)
      const int64_t run = std::min<int64_t>(n0 - idx[0], hi - i);
      T* b = B_ + ob;
      const T* a = A_ + oa;
      if (betaIsZero)
        for (int64_t r = 0; r < run; ++r) b[r] = alpha_ * a[r * sa0];
      else
        for (int64_t r = 0; r < run; ++r) b[r] = alpha_ * a[r * sa0] + beta_ * b[r];
      i += run;
      oa += run * sa0;
      ob += run;
      idx[0] += run;
      for (int j = 0; j < dim_ && idx[j] == ext_[j]; ++j) {  // carry
        oa -= idx[j] * sa_[j];
        ob -= idx[j] * sb_[j];
        idx[j] = 0;
        if (j + 1 < dim_) {
          idx[j + 1]++;
          oa += sa_[j + 1];
          ob += sb_[j + 1];
        }
      }
    }
  }

  int dim_;
  const T* A_;
  T* B_;
  T alpha_, beta_;
  int numThreads_;
  int64_t total_ = 0;
  std::vector<int64_t> ext_, sa_, sb_;
  std::vector<int> threadIds_;
  std::mutex mu_;
};

// HPTT declares create_plan as overloads per element type (so literal 0 / 1.0
// scalars convert), not as a template.
inline std::shared_ptr<Transpose<float>> create_plan(
    const int* perm, const int dim, const float alpha, const float* A, const int* sizeA,
    const int* outerSizeA, const float beta, float* B, const int* outerSizeB,
    const SelectionMethod, const int numThreads, const int* /*threadIds*/ = nullptr,
    const bool /*useRowMajor*/ = false) {
  return std::make_shared<Transpose<float>>(sizeA, perm, outerSizeA, outerSizeB, dim, A, alpha,
                                            B, beta, numThreads);
}

inline std::shared_ptr<Transpose<double>> create_plan(
    const int* perm, const int dim, const double alpha, const double* A, const int* sizeA,
    const int* outerSizeA, const double beta, double* B, const int* outerSizeB,
    const SelectionMethod, const int numThreads, const int* /*threadIds*/ = nullptr,
    const bool /*useRowMajor*/ = false) {
  return std::make_shared<Transpose<double>>(sizeA, perm, outerSizeA, outerSizeB, dim, A, alpha,
                                             B, beta, numThreads);
}

}  // namespace hptt
