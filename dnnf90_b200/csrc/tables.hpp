// tables.hpp - multi-index table sets (the product's own build of them).
//
// Restates init_hod_tables (lib/multi_index_bell_module.f90:128-351) and
// build_tanh_poly (:406-429): the graded combinations-with-replacement
// enumeration, the downward closure of seed multi-indices, the forward
// convolution lists fq_* and the adjoint pair lists pair_*, in exactly the
// reference's order, because the slot order is part of the interface
// (dnnf90_alpha, every t[] and seed[] array) and the list order fixes the
// summation order of the FP64 path.
//
// On top of the reference lists it derives the device program of the Bell
// kernels: which B_{alpha,q} values are kept in the per-neuron state and
// where (slot), and the packed (ib, id) term words.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace dnnf90 {

struct TableSet {
  int d0 = 0, k = 0, na = 0;
  int iact = 0;                  // 0 tanh, 1 sin, 2 erf, 3 J0, 4 J1
  std::vector<int> alpha;        // [na][d0]
  std::vector<int> deg;          // [na]
  std::vector<int> ind_e1;       // [d0], 0-based slot or -1
  // forward lists, reference order: for ia = 1..na-1, q = 2..deg(ia)
  std::vector<int> fq_start;     // [na][k+1] (q index), start into fq_*
  std::vector<int> fq_num;       // [na][k+1]
  std::vector<int> fq_ib, fq_id; // 0-based slots
  std::vector<double> fq_c;      // C(alpha,beta)/q
  // adjoint lists: for ib = 1..na-1, ia >= ib
  std::vector<int> pair_start, pair_num;  // [na]
  std::vector<int> pair_ia, pair_id;      // 0-based
  std::vector<double> pair_binom;
  std::vector<double> tpc;       // tanh polynomials, tpc(i,q) at q*(k+3)+i
  int nbell = 0;                 // "Bell table terms" count (diagnostic)

  // device program derived from the lists
  std::vector<int> bslot;        // [na][k+1]: state slot of B_{ia,q} or -1
  int nslot = 0;                 // per-neuron state slots (q >= 2, deg < k)

  int fq_at(int ia, int q) const { return fq_start[ia * (k + 1) + q]; }
  int fq_len(int ia, int q) const { return fq_num[ia * (k + 1) + q]; }
  int find(const int *a) const;  // slot of multi-index a, or -1
};

// Builds a table set; returns an empty string on success or the reason the
// arguments are refused (the reference's table_args_ok plus size limits).
std::string build_tables(int d0, int k, int nseed, const int *seeds,
                         TableSet &out);

}  // namespace dnnf90
