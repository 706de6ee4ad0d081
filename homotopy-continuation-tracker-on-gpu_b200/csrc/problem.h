// problem.h -- host-side problem description: YAML subset, reference text
// files, table validation and compilation into device term words.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

#include "ghc_internal.h"

namespace ghc {

struct P2CTerm {
  int k;
  double coef;
  std::vector<int> fac;  // parameter indices (0-based), with repetition
};

// Index tables a drop-in wrapper was handed that differ from the loaded ones: the caller's raw
// tables, their compiled form (host copies, which stay alive while their upload is queued) and the
// device copies (hx terms, hx offsets, ht terms, ht offsets).
struct CallerTables {
  std::vector<int32_t> hx_raw, ht_raw;
  std::vector<uint64_t> hx_terms, ht_terms;
  std::vector<uint16_t> hx_off, ht_off;
  void* dev[4] = {nullptr, nullptr, nullptr, nullptr};
  void release();
};

struct DeviceTables {
  int device = -1;
  uint64_t* hx_terms = nullptr;
  uint16_t* hx_off = nullptr;
  uint64_t* ht_terms = nullptr;
  uint16_t* ht_off = nullptr;
  // P2C expression tables
  int* t_k = nullptr;
  double* t_coef = nullptr;
  int* t_nf = nullptr;
  int* t_fac_off = nullptr;
  int* t_fac = nullptr;
  int* k_off = nullptr;
  // drop-in scratch (grow-only)
  void* scratch = nullptr;
  size_t scratch_bytes = 0;
  // ghc_solve_host: grow-only device arena and the handle's own non-blocking stream
  void* solve_arena = nullptr;
  size_t solve_bytes = 0;
  void* solve_stream = nullptr;
  int* counter = nullptr;
  CallerTables caller;
};

struct Problem {
  std::string name, print_name, type, ransac;
  int kind = KIND_P2C;
  int N = 0, P = 0, M = 0, K = 0, paths = 0;
  int Tx = 0, Px = 0, Tt = 0, Pt = 0;
  int max_steps = 0, max_corr = 0, incr = 0;
  std::vector<double> start_params, target_params;  // [P+1] complex
  std::vector<double> start_sols;                   // [paths][N] complex
  std::vector<int32_t> hx_raw, ht_raw;
  // compiled tables
  std::vector<uint64_t> hx_terms, ht_terms;
  std::vector<uint16_t> hx_off, ht_off;
  // P2C coefficient expressions (p2c_terms.txt), grouped by k
  bool has_terms = false;
  std::vector<P2CTerm> p2c;
  std::vector<int> p2c_k_off;  // [M+1]
  // launch tuning per precision (0: FP64, 1: FP32), set by ghc_autotune / ghc_set_tuning:
  // compiled register-budget variant and H_x walk (-1: flat_eval_pays() decides)
  int tune_variant[2] = {0, 0};
  int tune_flat[2] = {-1, -1};
  DeviceTables dev;
  uint64_t uid = 0;  // unique per loaded handle (set by load_problem; never reused in a process)
  ~Problem();
};

// the problem's tuning into a launch of `precision` (the FP32 phase's choices for mixed)
inline void apply_tuning(const Problem& pb, int precision, TrackParams& p) {
  const int heur = flat_eval_pays(pb.hx_off.data(), pb.N);
  const int f64 = pb.tune_flat[0] >= 0 ? pb.tune_flat[0] : heur;
  const int f32 = pb.tune_flat[1] >= 0 ? pb.tune_flat[1] : heur;
  const bool fp32 = precision == PREC_FP32;
  p.variant = fp32 ? pb.tune_variant[1] : pb.tune_variant[0];
  p.flat_eval = fp32 ? f32 : f64;
  p.variant_f32 = pb.tune_variant[1];
  p.flat_eval_f32 = f32;
}

// All return GHC_OK or a negative error code and set the thread's error message.
int load_problem(const std::string& root, const std::string& name, Problem& pb);
int compile_tables(const std::vector<int32_t>& hx, const std::vector<int32_t>& ht, const Problem& shape,
                   std::vector<uint64_t>& hx_terms, std::vector<uint16_t>& hx_off, std::vector<uint64_t>& ht_terms,
                   std::vector<uint16_t>& ht_off);
int p2c_host(const Problem& pb, const double* start, const double* target, double* hx, double* ht, int exact_ht);
int ensure_device(Problem& pb);
void* scratch(Problem& pb, size_t bytes);

void set_error(const std::string& msg);

}  // namespace ghc
