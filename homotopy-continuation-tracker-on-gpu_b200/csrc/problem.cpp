// problem.cpp -- problem loading, validation, table compilation and host P2C.
//
// File formats follow the reference readers (GPU-HC/magmaHC/Data_Reader.cpp:91-225):
//   start_params.txt / target_params.txt  whitespace "re im" pairs, P of them; slot P := 1
//   start_sols.txt                        "re im" per line, N lines per path, paths in order
//   dHdx_indx.txt / dHdt_indx.txt         whitespace integers in file order
// and the YAML keys of GPU_HC_Solver.cpp:44-66 (flat "key: value" subset with
// '#' comments and the "%YAML:1.0" header, which is all the shipped files use).
#include "problem.h"

#include <cuda_runtime.h>

#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstring>
#include <fstream>
#include <map>
#include <sstream>

#include "../../include/ghc.h"

namespace ghc {

namespace {
thread_local std::string g_err;

bool read_yaml(const std::string& path, std::map<std::string, std::string>& kv) {
  std::ifstream f(path);
  if (!f) return false;
  std::string line;
  while (std::getline(f, line)) {
    const size_t h = line.find('#');
    if (h != std::string::npos) line = line.substr(0, h);
    if (!line.empty() && line[0] == '%') continue;
    const size_t c = line.find(':');
    if (c == std::string::npos) continue;
    std::string key = line.substr(0, c), val = line.substr(c + 1);
    auto trim = [](std::string s) {
      const size_t a = s.find_first_not_of(" \t\r\n");
      if (a == std::string::npos) return std::string();
      const size_t b = s.find_last_not_of(" \t\r\n");
      return s.substr(a, b - a + 1);
    };
    key = trim(key);
    val = trim(val);
    if (!key.empty()) kv[key] = val;
  }
  return true;
}

bool get_int(const std::map<std::string, std::string>& kv, const char* key, int& out) {
  auto it = kv.find(key);
  if (it == kv.end()) return false;
  char* end = nullptr;
  const long v = std::strtol(it->second.c_str(), &end, 10);
  if (end == it->second.c_str() || *end != '\0') return false;
  out = (int)v;
  return true;
}

// "re im" pairs; returns the number of complete pairs read
long read_pairs(const std::string& path, std::vector<double>& out, bool& ok) {
  std::ifstream f(path);
  ok = (bool)f;
  out.clear();
  if (!f) return 0;
  double a, b;
  while (f >> a >> b) {
    out.push_back(a);
    out.push_back(b);
  }
  return (long)out.size() / 2;
}

bool read_ints(const std::string& path, std::vector<int32_t>& out) {
  std::ifstream f(path);
  if (!f) return false;
  out.clear();
  long long v;
  while (f >> v) out.push_back((int32_t)v);
  return f.eof();
}
}  // namespace

void set_error(const std::string& msg) { g_err = msg; }
const char* last_error() { return g_err.c_str(); }

void CallerTables::release() {
  for (void*& d : dev) {
    if (d) cudaFree(d);
    d = nullptr;
  }
}

Problem::~Problem() {
  if (dev.device >= 0) {
    int cur = 0;
    cudaGetDevice(&cur);
    cudaSetDevice(dev.device);
    cudaFree(dev.hx_terms);
    cudaFree(dev.hx_off);
    cudaFree(dev.ht_terms);
    cudaFree(dev.ht_off);
    cudaFree(dev.t_k);
    cudaFree(dev.t_coef);
    cudaFree(dev.t_nf);
    cudaFree(dev.t_fac_off);
    cudaFree(dev.t_fac);
    cudaFree(dev.k_off);
    cudaFree(dev.scratch);
    cudaFree(dev.solve_arena);
    if (dev.solve_stream) cudaStreamDestroy((cudaStream_t)dev.solve_stream);
    cudaFree(dev.counter);
    dev.caller.release();
    cudaSetDevice(cur);
  }
}

int compile_tables(const std::vector<int32_t>& hx, const std::vector<int32_t>& ht, const Problem& s,
                   std::vector<uint64_t>& hx_terms, std::vector<uint16_t>& hx_off, std::vector<uint64_t>& ht_terms,
                   std::vector<uint16_t>& ht_off) {
  const int N = s.N, Tx = s.Tx, Px = s.Px, Tt = s.Tt, Pt = s.Pt;
  const bool ph = s.kind == KIND_PH;
  const int n_coef_slots = ph ? 2 : 1;            // parameter pair (PH) or coefficient index (P2C)
  const int coef_limit = ph ? s.P + 1 : s.M + 1;  // valid index range
  if ((long)hx.size() != (long)N * N * Tx * Px || (long)ht.size() != (long)N * Tt * Pt) {
    set_error("table size does not match the YAML shape");
    return GHC_ERR_FORMAT;
  }
  if (Px - 1 - n_coef_slots > kMaxVarsPerTerm || Pt - 1 - n_coef_slots > kMaxVarsPerTerm || Px < 2 || Pt < 2) {
    set_error("unsupported number of parts per term");
    return GHC_ERR_RANGE;
  }
  auto get_hx = [&](int r, int i, int j, int q) -> int32_t {
    if (!ph) return hx[(((size_t)r * N + i) * Tx + j) * Px + q];
    return hx[(((size_t)i * Tx * Px) + (size_t)j * Px + q) * N + r];
  };
  auto get_ht = [&](int r, int j, int q) -> int32_t {
    if (!ph) return ht[((size_t)r * Tt + j) * Pt + q];
    return ht[((size_t)j * Pt + q) * N + r];
  };
  auto encode = [&](const int32_t* e, int parts, uint64_t& w) -> int {
    const int scale = e[0];
    if (scale < -128 || scale > 127) {
      set_error("term scale out of the int8 range");
      return GHC_ERR_RANGE;
    }
    w = (uint64_t)(uint8_t)(int8_t)scale;
    for (int c = 0; c < n_coef_slots; ++c) {
      if (e[1 + c] < 0 || e[1 + c] >= coef_limit) {
        set_error("coefficient/parameter index out of range in a table");
        return GHC_ERR_RANGE;
      }
    }
    if (ph) {
      w |= (uint64_t)(e[1] & 0x3f) << 11;
      w |= (uint64_t)(e[2] & 0x3f) << 17;
    } else {
      if (e[1] > 1023) {
        set_error("coefficient index above 1023");
        return GHC_ERR_RANGE;
      }
      w |= (uint64_t)e[1] << 11;
    }
    // every variable slot of the reference's term, slot N (the constant 1) included, so
    // that all terms of one table have the same number of factors
    int nv = 0;
    for (int q = 1 + n_coef_slots; q < parts; ++q) {
      const int v = e[q];
      if (v < 0 || v > N || v > 31) {
        set_error("variable index out of range in a table");
        return GHC_ERR_RANGE;
      }
      w |= (uint64_t)v << (24 + 5 * nv);
      ++nv;
    }
    w |= (uint64_t)nv << 8;
    return GHC_OK;
  };
  hx_terms.clear();
  ht_terms.clear();
  hx_off.assign((size_t)N * N + 1, 0);
  ht_off.assign((size_t)N + 1, 0);
  int32_t e[16];
  for (int r = 0; r < N; ++r) {
    for (int i = 0; i < N; ++i) {
      hx_off[(size_t)r * N + i] = (uint16_t)hx_terms.size();
      for (int j = 0; j < Tx; ++j) {
        for (int q = 0; q < Px; ++q) e[q] = get_hx(r, i, j, q);
        if (e[0] == 0) continue;
        uint64_t w;
        const int rc = encode(e, Px, w);
        if (rc) return rc;
        hx_terms.push_back(w | (uint64_t)i << 59);
      }
      // the entry's last term ends its sum in the row-wise walk
      if (hx_terms.size() > hx_off[(size_t)r * N + i]) hx_terms.back() |= kTermLast;
    }
  }
  hx_off[(size_t)N * N] = (uint16_t)hx_terms.size();
  for (int r = 0; r < N; ++r) {
    ht_off[r] = (uint16_t)ht_terms.size();
    for (int j = 0; j < Tt; ++j) {
      for (int q = 0; q < Pt; ++q) e[q] = get_ht(r, j, q);
      if (e[0] == 0) continue;
      uint64_t w;
      const int rc = encode(e, Pt, w);
      if (rc) return rc;
      ht_terms.push_back(w);
    }
  }
  ht_off[N] = (uint16_t)ht_terms.size();
  // Row-interleaved storage: term k of row r at k * N + r, rows padded with zero
  // words to the longest row, so the lanes of a sub-warp (one row each) read
  // consecutive words of shared memory.  The CSR offsets keep their meaning:
  // term j of row r (hx_off[r N] <= j < hx_off[(r+1) N]) sits at (j - hx_off[r N]) N + r.
  auto interleave = [&](std::vector<uint64_t>& terms, const std::vector<uint16_t>& off, int per_row) {
    int longest = 0;
    for (int r = 0; r < N; ++r) longest = std::max(longest, off[(size_t)(r + 1) * per_row] - off[(size_t)r * per_row]);
    std::vector<uint64_t> out((size_t)longest * N, 0);
    for (int r = 0; r < N; ++r)
      for (int k = off[(size_t)r * per_row]; k < off[(size_t)(r + 1) * per_row]; ++k)
        out[(size_t)(k - off[(size_t)r * per_row]) * N + r] = terms[k];
    terms.swap(out);
  };
  // Balanced H_x walk: the entries (row, column) are dealt to the W lanes of a sub-warp, longest
  // first, each to the lane with the fewest terms so far (lowest lane on ties); a lane walks its
  // entries' terms, each entry's in table order, so every sum is formed exactly as in the row-wise
  // walk, only by another lane.  Words carry the entry's destination (row, slot among the row's
  // non-zero entries).  Stored after the row-interleaved block, term q of lane l at q * W + l.
  const int W = subwarp_width(N);
  std::vector<uint64_t> lane_words;
  std::vector<int> lane_len(W, 0);
  const bool balanced = balanced_walk_built(N) && Px - 1 - n_coef_slots <= kMaxVarsBalanced;
  if (balanced) {
    struct Entry {
      int r, slot, beg, end;
    };
    std::vector<Entry> entries;
    for (int r = 0; r < N; ++r) {
      int slot = 0;
      for (int i = 0; i < N; ++i) {
        const int beg = hx_off[(size_t)r * N + i], end = hx_off[(size_t)r * N + i + 1];
        if (end > beg) entries.push_back({r, slot++, beg, end});
      }
    }
    std::stable_sort(entries.begin(), entries.end(),
                     [](const Entry& a, const Entry& b) { return a.end - a.beg > b.end - b.beg; });
    std::vector<std::vector<int>> lists(W);
    for (int e = 0; e < (int)entries.size(); ++e) {
      int best = 0;
      for (int l = 1; l < W; ++l)
        if (lane_len[l] < lane_len[best]) best = l;
      lists[best].push_back(e);
      lane_len[best] += entries[e].end - entries[e].beg;
    }
    const int longest = *std::max_element(lane_len.begin(), lane_len.end());
    lane_words.assign((size_t)longest * W, 0);
    for (int l = 0; l < W; ++l) {
      int q = 0;
      for (int e : lists[l]) {
        const Entry& en = entries[e];
        for (int j = en.beg; j < en.end; ++j)
          lane_words[(size_t)(q++) * W + l] = hx_terms[j] | (uint64_t)en.r << 49 | (uint64_t)en.slot << 54;
      }
    }
  }
  interleave(hx_terms, hx_off, N);
  interleave(ht_terms, ht_off, 1);
  hx_off.push_back(balanced ? (uint16_t)hx_terms.size() : kNoLanes);
  for (int l = 0; l < W; ++l) hx_off.push_back((uint16_t)lane_len[l]);
  hx_terms.insert(hx_terms.end(), lane_words.begin(), lane_words.end());
  if (hx_terms.size() > 60000 || ht_terms.size() > 60000) {
    set_error("too many terms");
    return GHC_ERR_LIMIT;
  }
  return GHC_OK;
}

int load_problem(const std::string& root, const std::string& name, Problem& pb) {
  const std::string dir = root + "/" + name;
  std::map<std::string, std::string> kv;
  if (!read_yaml(dir + "/gpuhc_settings.yaml", kv)) {
    set_error("cannot read " + dir + "/gpuhc_settings.yaml");
    return GHC_ERR_IO;
  }
  static std::atomic<uint64_t> next_uid{1};
  pb.uid = next_uid++;
  pb.name = name;
  pb.print_name = kv.count("problem_print_out_name") ? kv["problem_print_out_name"] : name;
  pb.type = kv.count("GPUHC_Type") ? kv["GPUHC_Type"] : "";
  pb.ransac = kv.count("RANSAC_Dataset") ? kv["RANSAC_Dataset"] : "None";
  if (pb.type != "P2C" && pb.type != "PH") {
    set_error("GPUHC_Type must be P2C or PH");
    return GHC_ERR_FORMAT;
  }
  pb.kind = pb.type == "P2C" ? KIND_P2C : KIND_PH;
  bool ok = get_int(kv, "GPUHC_Max_Steps", pb.max_steps) && get_int(kv, "GPUHC_Max_Correction_Steps", pb.max_corr) &&
            get_int(kv, "GPUHC_Num_Of_Steps_to_Increase_Delta_t", pb.incr) && get_int(kv, "Num_Of_Vars", pb.N) &&
            get_int(kv, "Num_Of_Params", pb.P) && get_int(kv, "Num_Of_Tracks", pb.paths) &&
            get_int(kv, "dHdx_Max_Terms", pb.Tx) && get_int(kv, "dHdx_Max_Parts", pb.Px) &&
            get_int(kv, "dHdt_Max_Terms", pb.Tt) && get_int(kv, "dHdt_Max_Parts", pb.Pt) &&
            get_int(kv, "Max_Order_Of_T", pb.K);
  if (pb.kind == KIND_P2C) ok = ok && get_int(kv, "Num_Of_Coeffs_From_Params", pb.M);
  if (!ok) {
    set_error("missing or non-integer key in gpuhc_settings.yaml");
    return GHC_ERR_FORMAT;
  }
  if (pb.N < 1 || pb.N > kMaxN || pb.P < 0 || pb.paths < 1 || pb.Tx < 1 || pb.Tt < 1 || pb.K < 0 || pb.K > 8 ||
      pb.M < 0 || pb.M > 1023 || pb.P > 62 * (pb.kind == KIND_PH) + 100000 * (pb.kind == KIND_P2C)) {
    set_error("problem sizes out of the supported range (N <= 32)");
    return GHC_ERR_RANGE;
  }
  // parameters (slot P = 1)
  std::vector<double> v;
  for (int which = 0; which < 2; ++which) {
    const std::string f = dir + (which == 0 ? "/start_params.txt" : "/target_params.txt");
    const long n = read_pairs(f, v, ok);
    std::vector<double>& dst = which == 0 ? pb.start_params : pb.target_params;
    dst.assign(2 * (size_t)(pb.P + 1), 0.0);
    if (!ok) {
      if (which == 1) {  // a problem may ship no target (targets come from the caller)
        dst[2 * pb.P] = 1.0;
        continue;
      }
      set_error("cannot read " + f);
      return GHC_ERR_IO;
    }
    // The reference reads as many pairs as the file holds (Data_Reader.cpp:140-149, 166-175) and
    // leaves the rest of its parameter array unset; uncalibrated_trifocal_rel_pos_CH ships 18 of
    // its 24 target parameters.  Missing trailing parameters are 0 here (deterministic), extra
    // pairs beyond Num_Of_Params are ignored.
    const long use = std::min<long>(n, pb.P);
    std::copy(v.begin(), v.begin() + 2 * use, dst.begin());
    dst[2 * pb.P] = 1.0;
    dst[2 * pb.P + 1] = 0.0;
  }
  // start solutions
  {
    const long n = read_pairs(dir + "/start_sols.txt", v, ok);
    if (!ok) {
      set_error("cannot read start_sols.txt");
      return GHC_ERR_IO;
    }
    if (n < (long)pb.paths * pb.N) {
      set_error("start_sols.txt holds fewer than Num_Of_Tracks * Num_Of_Vars values");
      return GHC_ERR_FORMAT;
    }
    pb.start_sols.assign(v.begin(), v.begin() + 2 * (size_t)pb.paths * pb.N);
  }
  if (!read_ints(dir + "/dHdx_indx.txt", pb.hx_raw) || !read_ints(dir + "/dHdt_indx.txt", pb.ht_raw)) {
    set_error("cannot read or parse dHdx_indx.txt / dHdt_indx.txt");
    return GHC_ERR_IO;
  }
  int rc = compile_tables(pb.hx_raw, pb.ht_raw, pb, pb.hx_terms, pb.hx_off, pb.ht_terms, pb.ht_off);
  if (rc) return rc;
  // optional coefficient expressions
  std::ifstream tf(dir + "/p2c_terms.txt");
  if (tf && pb.kind == KIND_P2C) {
    std::string line;
    int M = -1, K = -1, P = -1;
    std::vector<std::vector<P2CTerm>> byk;
    while (std::getline(tf, line)) {
      if (line.empty() || line[0] == '#') continue;
      std::istringstream ls(line);
      if (M < 0) {
        ls >> M >> K >> P;
        if (M != pb.M || K != pb.K || P != pb.P) {
          set_error("p2c_terms.txt header does not match the YAML");
          return GHC_ERR_FORMAT;
        }
        byk.assign(M, {});
        continue;
      }
      P2CTerm t;
      long long num, den;
      int nf;
      if (!(ls >> t.k >> num >> den >> nf) || t.k < 0 || t.k >= M || den == 0 || nf < 0 || nf > K) {
        set_error("malformed p2c_terms.txt line");
        return GHC_ERR_FORMAT;
      }
      t.coef = (double)num / (double)den;
      t.fac.resize(nf);
      for (int q = 0; q < nf; ++q) {
        if (!(ls >> t.fac[q]) || t.fac[q] < 0 || t.fac[q] >= P) {
          set_error("malformed p2c_terms.txt factor");
          return GHC_ERR_FORMAT;
        }
      }
      byk[t.k].push_back(t);
    }
    pb.p2c.clear();
    pb.p2c_k_off.assign((size_t)pb.M + 1, 0);
    for (int k = 0; k < pb.M; ++k) {
      pb.p2c_k_off[k] = (int)pb.p2c.size();
      for (auto& t : byk[k]) pb.p2c.push_back(t);
    }
    pb.p2c_k_off[pb.M] = (int)pb.p2c.size();
    pb.has_terms = M >= 0;
  }
  return GHC_OK;
}

// c_k(t) = sum_terms coef * prod_j (q_j + t d_j), expanded in ascending powers of t
int p2c_host(const Problem& pb, const double* start, const double* target, double* hx, double* ht, int exact_ht) {
  if (pb.kind != KIND_P2C || !pb.has_terms) {
    set_error("problem has no coefficient expressions (p2c_terms.txt)");
    return GHC_ERR_NOP2C;
  }
  const int M = pb.M, K = pb.K;
  std::vector<double> poly(2 * (K + 1)), nxt(2 * (K + 1)), acc(2 * (K + 1));
  for (int k = 0; k <= M; ++k) {
    std::fill(acc.begin(), acc.end(), 0.0);
    if (k == M) {
      acc[0] = 1.0;
    } else {
      for (int ti = pb.p2c_k_off[k]; ti < pb.p2c_k_off[k + 1]; ++ti) {
        const P2CTerm& t = pb.p2c[ti];
        std::fill(poly.begin(), poly.end(), 0.0);
        poly[0] = t.coef;
        int deg = 0;
        for (int j : t.fac) {
          const double qr = start[2 * j], qi = start[2 * j + 1];
          const double dr = target[2 * j] - qr, di = target[2 * j + 1] - qi;
          std::fill(nxt.begin(), nxt.end(), 0.0);
          for (int e = 0; e <= deg; ++e) {
            const double pr = poly[2 * e], pi = poly[2 * e + 1];
            nxt[2 * e] += pr * qr - pi * qi;
            nxt[2 * e + 1] += pr * qi + pi * qr;
            nxt[2 * (e + 1)] += pr * dr - pi * di;
            nxt[2 * (e + 1) + 1] += pr * di + pi * dr;
          }
          ++deg;
          poly.swap(nxt);
        }
        for (int e = 0; e <= K; ++e) {
          acc[2 * e] += poly[2 * e];
          acc[2 * e + 1] += poly[2 * e + 1];
        }
      }
    }
    for (int e = 0; e <= K; ++e) {
      hx[2 * ((size_t)k * (K + 1) + e)] = acc[2 * e];
      hx[2 * ((size_t)k * (K + 1) + e) + 1] = acc[2 * e + 1];
    }
    for (int e = 0; e < K; ++e) {
      double r = (e + 1) * acc[2 * (e + 1)], i = (e + 1) * acc[2 * (e + 1) + 1];
      if (k == M) {
        r = (e == 0 && !exact_ht) ? 1.0 : 0.0;
        i = 0.0;
      }
      ht[2 * ((size_t)k * K + e)] = r;
      ht[2 * ((size_t)k * K + e) + 1] = i;
    }
  }
  return GHC_OK;
}

namespace {
template <typename T>
int upload(T** dst, const std::vector<T>& src) {
  const size_t n = std::max<size_t>(src.size(), 1);
  if (cudaMalloc((void**)dst, n * sizeof(T)) != cudaSuccess) return GHC_ERR_CUDA;
  if (!src.empty() && cudaMemcpy(*dst, src.data(), src.size() * sizeof(T), cudaMemcpyHostToDevice) != cudaSuccess)
    return GHC_ERR_CUDA;
  return GHC_OK;
}
}  // namespace

int ensure_device(Problem& pb) {
  int cur = 0;
  if (cudaGetDevice(&cur) != cudaSuccess) {
    set_error("no CUDA device");
    return GHC_ERR_CUDA;
  }
  if (pb.dev.device == cur) return GHC_OK;
  if (pb.dev.device >= 0) {
    set_error("problem handle already bound to another device");
    return GHC_ERR_ARG;
  }
  int rc = upload(&pb.dev.hx_terms, pb.hx_terms) | upload(&pb.dev.hx_off, pb.hx_off) |
           upload(&pb.dev.ht_terms, pb.ht_terms) | upload(&pb.dev.ht_off, pb.ht_off);
  if (pb.has_terms) {
    std::vector<int> tk, tnf, toff, tfac;
    std::vector<double> tc;
    toff.push_back(0);
    for (auto& t : pb.p2c) {
      tk.push_back(t.k);
      tc.push_back(t.coef);
      tnf.push_back((int)t.fac.size());
      for (int f : t.fac) tfac.push_back(f);
      toff.push_back((int)tfac.size());
    }
    rc |= upload(&pb.dev.t_k, tk) | upload(&pb.dev.t_coef, tc) | upload(&pb.dev.t_nf, tnf) |
          upload(&pb.dev.t_fac_off, toff) | upload(&pb.dev.t_fac, tfac) | upload(&pb.dev.k_off, pb.p2c_k_off);
  }
  if (cudaMalloc((void**)&pb.dev.counter, sizeof(int)) != cudaSuccess) rc = GHC_ERR_CUDA;
  if (rc) {
    set_error(std::string("device upload failed: ") + cudaGetErrorString(cudaGetLastError()));
    return GHC_ERR_CUDA;
  }
  pb.dev.device = cur;
  return GHC_OK;
}

void* scratch(Problem& pb, size_t bytes) {
  if (bytes <= pb.dev.scratch_bytes) return pb.dev.scratch;
  cudaFree(pb.dev.scratch);
  pb.dev.scratch = nullptr;
  pb.dev.scratch_bytes = 0;
  if (cudaMalloc(&pb.dev.scratch, bytes) != cudaSuccess) return nullptr;
  pb.dev.scratch_bytes = bytes;
  return pb.dev.scratch;
}

}  // namespace ghc
