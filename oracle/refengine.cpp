// ORACLE — test/benchmark infrastructure only (never linked by the product).
// A reference-shaped CPU engine: the algorithms and the parallel structure of
// FalconDB's rayon operators, restated in C++ because the Rust crate cannot be
// built here.  bench.py times it as the CPU baseline ("port") on the GPU box's
// host cores.  It mirrors, per query:
//   * 65,536-row batches (Table::MAX_BATCH_ROWS, storage/table.rs:339);
//   * SUM / COUNT(DISTINCT): execute_agg_only folds batches in parallel
//     (aggregate.rs:1496-1515), SUM with 8 f64 lanes (sum_lanes 1557-1590),
//     COUNT(DISTINCT) via per-batch present_codes (3167-3200);
//   * COUNT(*) WHERE: a serial loop over batches, each an AVX2 compare ->
//     movemask mask (cmp_f64_avx2, expr.rs:865-902) and a popcount (db.rs:1453-1458);
//   * ORDER BY .. LIMIT k: a serial loop over batches, each reduced by the
//     bounded-buffer top_k_ascending, then the merged parts sorted again
//     (sort.rs:59-115, 564-599);
//   * filter -> GROUP BY dept: parallel per-batch mask + gather
//     (select.rs:105-160), then parallel chunked accumulation into per-chunk
//     states and a serial merge (fast_utf8_gb, aggregate.rs:619-836);
//   * joins: serial build of the chained IntHashTable + Bloom filter, parallel
//     probe in units of >= 8192 rows (join.rs:297-375, 607-723, 1054-1482);
//   * int64 GROUP BY: per-batch hash maps in parallel, serial merge
//     (fast_i64_gb, aggregate.rs:840-912).
// Thread pool: a fixed team pulling work items from an atomic counter, the way
// rayon's work stealing spreads independent batches.
#include <algorithm>
#include <atomic>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <functional>
#include <thread>
#include <unordered_map>
#include <utility>
#include <vector>

#if defined(__x86_64__)
#include <immintrin.h>
#endif

namespace {

constexpr uint64_t kBatch = 65536;

void par_for(uint64_t items, int threads, const std::function<void(uint64_t)>& fn) {
  if (threads <= 1 || items <= 1) {
    for (uint64_t i = 0; i < items; ++i) fn(i);
    return;
  }
  std::atomic<uint64_t> next{0};
  std::vector<std::thread> team;
  const int nt = (int)std::min<uint64_t>((uint64_t)threads, items);
  for (int t = 0; t < nt; ++t)
    team.emplace_back([&] {
      for (;;) {
        const uint64_t i = next.fetch_add(1);
        if (i >= items) break;
        fn(i);
      }
    });
  for (auto& th : team) th.join();
}

double sum_lanes(const double* v, uint64_t n) {
  double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
  const uint64_t full = n / 8 * 8;
  for (uint64_t i = 0; i < full; i += 8)
    for (int l = 0; l < 8; ++l) acc[l] += v[i + l];
  double t = 0.0;
  for (int l = 0; l < 8; ++l) t += acc[l];
  for (uint64_t i = full; i < n; ++i) t += v[i];
  return t;
}

inline bool cmp_scalar(int op, double a, double b) {
  switch (op) {
    case 0: return a == b;
    case 1: return a != b;
    case 2: return a < b;
    case 3: return a <= b;
    case 4: return a > b;
    default: return a >= b;
  }
}

#if defined(__x86_64__)
__attribute__((target("avx2"))) void cmp_mask_avx2(const double* v, uint64_t n, int op, double lit,
                                                    uint64_t* mask) {
  const __m256d l = _mm256_set1_pd(lit);
  const uint64_t full = n / 4 * 4;
  for (uint64_t i = 0; i < full; i += 4) {
    const __m256d x = _mm256_loadu_pd(v + i);
    __m256d c;
    switch (op) {
      case 0: c = _mm256_cmp_pd(x, l, _CMP_EQ_OQ); break;
      case 1: c = _mm256_cmp_pd(x, l, _CMP_NEQ_UQ); break;
      case 2: c = _mm256_cmp_pd(x, l, _CMP_LT_OQ); break;
      case 3: c = _mm256_cmp_pd(x, l, _CMP_LE_OQ); break;
      case 4: c = _mm256_cmp_pd(x, l, _CMP_GT_OQ); break;
      default: c = _mm256_cmp_pd(x, l, _CMP_GE_OQ); break;
    }
    const uint64_t bits = (uint64_t)_mm256_movemask_pd(c);
    mask[i >> 6] |= bits << (i & 63);
  }
  for (uint64_t i = full; i < n; ++i)
    if (cmp_scalar(op, v[i], lit)) mask[i >> 6] |= 1ull << (i & 63);
}
#endif

void cmp_mask(const double* v, uint64_t n, int op, double lit, uint64_t* mask) {
  std::memset(mask, 0, ((n + 63) / 64) * 8);
#if defined(__x86_64__)
  if (__builtin_cpu_supports("avx2")) {
    cmp_mask_avx2(v, n, op, lit, mask);
    return;
  }
#endif
  for (uint64_t i = 0; i < n; ++i)
    if (cmp_scalar(op, v[i], lit)) mask[i >> 6] |= 1ull << (i & 63);
}

uint64_t nbatches(uint64_t n) { return (n + kBatch - 1) / kBatch; }

inline uint64_t ord_f64(double v) {
  uint64_t b;
  std::memcpy(&b, &v, 8);
  return (b >> 63) == 0 ? (b ^ (1ull << 63)) : ~b;
}

typedef std::pair<uint64_t, uint32_t> KP;

// top_k_ascending (sort.rs:564-599) over one batch; rows are batch-local.
std::vector<KP> top_k_ascending(const std::function<uint64_t(uint64_t)>& key, uint64_t n, uint32_t k) {
  const size_t cap = std::max<size_t>(2 * (size_t)k, 1024);
  std::vector<KP> buf;
  buf.reserve(cap);
  bool have = false;
  uint64_t worst = 0;
  for (uint64_t i = 0; i < n; ++i) {
    const uint64_t kk = key(i);
    if (have && kk > worst) continue;
    buf.emplace_back(kk, (uint32_t)i);
    if (buf.size() == cap) {
      std::nth_element(buf.begin(), buf.begin() + (k - 1), buf.end());
      worst = buf[k - 1].first;
      have = true;
      buf.resize(k);
    }
  }
  if (buf.size() > k) {
    std::nth_element(buf.begin(), buf.begin() + (k - 1), buf.end());
    buf.resize(k);
  }
  std::sort(buf.begin(), buf.end());
  return buf;
}

uint64_t bucket_with(uint64_t mask, int64_t key) {
  uint64_t h = (uint64_t)key;
  h ^= h >> 33;
  h *= 0xff51afd7ed558ccdull;
  h ^= h >> 33;
  return h & mask;
}

}  // namespace

extern "C" {

int ref_hardware_threads(void) {
  const unsigned n = std::thread::hardware_concurrency();
  return n ? (int)n : 1;
}

// SELECT SUM(score): execute_agg_only over batches in parallel.
double ref_sum_f64(const double* v, uint64_t n, int threads) {
  const uint64_t nb = nbatches(n);
  std::vector<double> part(nb, 0.0);
  par_for(nb, threads, [&](uint64_t b) {
    const uint64_t s = b * kBatch;
    part[b] = sum_lanes(v + s, std::min(kBatch, n - s));
  });
  double t = 0.0;
  for (double p : part) t += p;
  return t;
}

// SELECT COUNT(*) WHERE col op lit over a Float64 column: serial over batches.
uint64_t ref_count_cmp_f64(const double* v, uint64_t n, int op, double lit) {
  std::vector<uint64_t> mask(kBatch / 64);
  uint64_t total = 0;
  for (uint64_t s = 0; s < n; s += kBatch) {
    const uint64_t m = std::min(kBatch, n - s);
    cmp_mask(v + s, m, op, lit, mask.data());
    for (uint64_t w = 0; w < (m + 63) / 64; ++w) total += (uint64_t)__builtin_popcountll(mask[w]);
  }
  return total;
}

// COUNT(DISTINCT dept) over dictionary codes: present_codes per batch in
// parallel; out[d] = 1 if code d occurs anywhere.
void ref_present_codes(const uint32_t* codes, uint64_t n, uint32_t dict_len, int threads, uint8_t* out) {
  const uint64_t nb = nbatches(n);
  std::vector<std::vector<uint8_t>> part(nb);
  par_for(nb, threads, [&](uint64_t b) {
    std::vector<uint8_t> pr(dict_len, 0);
    const uint64_t s = b * kBatch, e = std::min(n, s + kBatch);
    for (uint64_t i = s; i < e; ++i)
      if (codes[i] < dict_len) pr[codes[i]] = 1;
    part[b] = std::move(pr);
  });
  std::memset(out, 0, dict_len);
  for (auto& pr : part)
    for (uint32_t d = 0; d < dict_len; ++d) out[d] |= pr[d];
}

// ORDER BY col [DESC] LIMIT k, serial over batches then a merged re-sort.
uint64_t ref_topk(int dtype, const void* values, uint64_t n, uint32_t k, int desc, uint32_t* out) {
  std::vector<KP> parts;
  for (uint64_t s = 0; s < n; s += kBatch) {
    const uint64_t m = std::min(kBatch, n - s);
    std::function<uint64_t(uint64_t)> key;
    if (dtype == 2) {
      const double* v = static_cast<const double*>(values) + s;
      key = [v, desc](uint64_t i) { const uint64_t x = ord_f64(v[i]); return desc ? ~x : x; };
    } else {
      const int64_t* v = static_cast<const int64_t*>(values) + s;
      key = [v, desc](uint64_t i) { const uint64_t x = (uint64_t)v[i] ^ (1ull << 63); return desc ? ~x : x; };
    }
    for (const KP& p : top_k_ascending(key, m, k)) parts.emplace_back(p.first, (uint32_t)(p.second + s));
  }
  std::sort(parts.begin(), parts.end());
  const uint64_t o = std::min<uint64_t>(k, parts.size());
  for (uint64_t i = 0; i < o; ++i) out[i] = parts[i].second;
  return o;
}

// SELECT dept, COUNT(*), SUM(score), AVG(salary) WHERE score op lit GROUP BY dept.
// out arrays hold dict_len entries: rows, sum(score), sum(salary as f64).
void ref_filter_group_codes(const uint32_t* codes, const double* score, const int64_t* salary, uint64_t n,
                            uint32_t dict_len, int op, double lit, int threads, int64_t* rows, double* fsum,
                            double* isum) {
  // Step 1: execute_select — per batch mask + gather of the survivors.
  const uint64_t nb = nbatches(n);
  struct Sel {
    std::vector<uint32_t> c;
    std::vector<double> f;
    std::vector<int64_t> i;
  };
  std::vector<Sel> sel(nb);
  par_for(nb, threads, [&](uint64_t b) {
    const uint64_t s = b * kBatch, m = std::min(kBatch, n - s);
    std::vector<uint64_t> mask((m + 63) / 64);
    cmp_mask(score + s, m, op, lit, mask.data());
    Sel& o = sel[b];
    for (uint64_t w = 0; w < mask.size(); ++w) {
      uint64_t x = mask[w];
      while (x) {
        const uint64_t r = s + w * 64 + (uint64_t)__builtin_ctzll(x);
        x &= x - 1;
        o.c.push_back(codes[r]);
        o.f.push_back(score[r]);
        o.i.push_back(salary[r]);
      }
    }
  });
  // Step 2: fast_utf8_gb — chunks of >= 4096 rows accumulate in parallel into
  // per-chunk states; a serial merge combines them.
  struct Chunk {
    uint64_t b, s, e;
  };
  std::vector<Chunk> work;
  for (uint64_t b = 0; b < nb; ++b)
    for (uint64_t s = 0; s < sel[b].c.size(); s += 4096) work.push_back({b, s, std::min<uint64_t>(sel[b].c.size(), s + 4096)});
  struct State {
    std::vector<int64_t> rows;
    std::vector<double> fs, is;
  };
  std::vector<State> st(work.size());
  par_for(work.size(), threads, [&](uint64_t w) {
    const Chunk& ch = work[w];
    State& x = st[w];
    x.rows.assign(dict_len, 0);
    x.fs.assign(dict_len, 0.0);
    x.is.assign(dict_len, 0.0);
    const Sel& sb = sel[ch.b];
    for (uint64_t r = ch.s; r < ch.e; ++r) {
      const uint32_t g = sb.c[r];
      if (g >= dict_len) continue;
      x.rows[g]++;
      x.fs[g] += sb.f[r];
      x.is[g] += (double)sb.i[r];
    }
  });
  for (uint32_t g = 0; g < dict_len; ++g) {
    rows[g] = 0;
    fsum[g] = 0.0;
    isum[g] = 0.0;
  }
  for (const State& x : st)
    for (uint32_t g = 0; g < dict_len; ++g) {
      rows[g] += x.rows[g];
      fsum[g] += x.fs[g];
      isum[g] += x.is[g];
    }
}

// Hash join: serial build (IntHashTable, 2 buckets per row, LIFO chains, plus
// the 16-bit-per-key Bloom filter), parallel probe in units of >= 8192 rows.
// join_type 0 INNER 1 LEFT 2 SEMI 3 ANTI; results as orc_join_agg.
void ref_join_agg(const int64_t* bkeys, const int64_t* bpay, uint64_t nb, const int64_t* pkeys, const double* pval,
                  uint64_t np, int join_type, int threads, int64_t* out_count, int64_t* out_psum, double* out_vsum) {
  uint64_t buckets = 1;
  while (buckets < std::max<uint64_t>(nb * 2, 1)) buckets <<= 1;
  const uint64_t mask = buckets - 1;
  std::vector<uint32_t> head(buckets, 0xFFFFFFFFu), next(nb, 0xFFFFFFFFu);
  uint64_t bloom_bits = 64;
  while (bloom_bits < std::max<uint64_t>(nb, 1) * 16) bloom_bits <<= 1;
  std::vector<uint64_t> bloom(bloom_bits / 64, 0);
  const uint64_t bmask = bloom.size() - 1;
  auto hash = [](int64_t k) {
    uint64_t h = (uint64_t)k;
    h ^= h >> 33;
    h *= 0xff51afd7ed558ccdull;
    h ^= h >> 33;
    return h;
  };
  for (uint64_t r = 0; r < nb; ++r) {
    const uint64_t b = bucket_with(mask, bkeys[r]);
    next[r] = head[b];
    head[b] = (uint32_t)r;
    const uint64_t h1 = hash(bkeys[r]), h2 = ((h1 << 32) | (h1 >> 32)) | 1;
    bloom[(h1 >> 6) & bmask] |= 1ull << (h1 & 63);
    bloom[(h2 >> 6) & bmask] |= 1ull << (h2 & 63);
  }
  const uint64_t unit = 8192;
  const uint64_t nu = (np + unit - 1) / unit;
  std::vector<int64_t> cnt(nu, 0), ps(nu, 0);
  std::vector<double> vs(nu, 0.0);
  par_for(nu, threads, [&](uint64_t u) {
    const uint64_t s = u * unit, e = std::min(np, s + unit);
    int64_t c = 0, p = 0;
    double v = 0.0;
    for (uint64_t i = s; i < e; ++i) {
      const int64_t k = pkeys[i];
      const uint64_t h1 = hash(k), h2 = ((h1 << 32) | (h1 >> 32)) | 1;
      int64_t m = 0, pp = 0;
      if (((bloom[(h1 >> 6) & bmask] >> (h1 & 63)) & 1ull) && ((bloom[(h2 >> 6) & bmask] >> (h2 & 63)) & 1ull)) {
        for (uint32_t r = head[bucket_with(mask, k)]; r != 0xFFFFFFFFu; r = next[r])
          if (bkeys[r] == k) {
            ++m;
            pp += bpay ? bpay[r] : 0;
          }
      }
      if (join_type <= 1) {
        c += (join_type == 1 && m == 0) ? 1 : m;
        p += pp;
      } else if ((join_type == 2) == (m != 0)) {
        ++c;
        if (pval) v += pval[i];
      }
    }
    cnt[u] = c;
    ps[u] = p;
    vs[u] = v;
  });
  int64_t c = 0, p = 0;
  double v = 0.0;
  for (uint64_t u = 0; u < nu; ++u) {
    c += cnt[u];
    p += ps[u];
    v += vs[u];
  }
  *out_count = c;
  *out_psum = p;
  *out_vsum = v;
}

// GROUP BY int64 key with COUNT/SUM/MIN/MAX: per-batch maps in parallel, then
// a serial merge into one map.  Returns the number of groups.
uint64_t ref_group_i64(const int64_t* keys, const double* vals, uint64_t n, int threads) {
  struct Acc {
    int64_t c = 0;
    double s = 0.0, mn = INFINITY, mx = -INFINITY;
  };
  const uint64_t nb = nbatches(n);
  std::vector<std::unordered_map<int64_t, Acc>> part(nb);
  par_for(nb, threads, [&](uint64_t b) {
    auto& m = part[b];
    const uint64_t s = b * kBatch, e = std::min(n, s + kBatch);
    m.reserve(e - s);
    for (uint64_t i = s; i < e; ++i) {
      Acc& a = m[keys[i]];
      a.c++;
      a.s += vals[i];
      a.mn = std::fmin(a.mn, vals[i]);
      a.mx = std::fmax(a.mx, vals[i]);
    }
  });
  std::unordered_map<int64_t, Acc> all;
  for (auto& m : part)
    for (auto& kv : m) {
      Acc& a = all[kv.first];
      a.c += kv.second.c;
      a.s += kv.second.s;
      a.mn = std::fmin(a.mn, kv.second.mn);
      a.mx = std::fmax(a.mx, kv.second.mx);
    }
  return all.size();
}

// SELECT col ORDER BY col [DESC] (no LIMIT): try_typed_sort's pair loop
// (sort.rs:270-287, 326-345: (order key, row) pairs of the non-NULL rows, NULL
// rows collected apart, serially), then the pairs sorted as tuples in parallel
// (sort_pairs_ord -> par_sort_unstable, sort.rs:692-698; here one std::sort
// per thread's run and parallel pairwise merges), then assemble (773-791).
void ref_sort(int dtype, const void* values, const uint64_t* validity, uint64_t n, int desc, int nulls_last,
              int threads, uint32_t* out) {
  typedef std::pair<uint64_t, uint32_t> P;
  std::vector<P> pairs;
  pairs.reserve(n);
  std::vector<uint32_t> nulls;
  for (uint64_t i = 0; i < n; ++i) {
    if (validity && !((validity[i >> 6] >> (i & 63)) & 1ull)) {
      nulls.push_back((uint32_t)i);
      continue;
    }
    uint64_t key = dtype == 2 ? ord_f64(static_cast<const double*>(values)[i])
                              : ((uint64_t)static_cast<const int64_t*>(values)[i] ^ (1ull << 63));
    pairs.emplace_back(desc ? ~key : key, (uint32_t)i);
  }
  const uint64_t m = pairs.size();
  const uint64_t runs = std::max<uint64_t>(1, std::min<uint64_t>((uint64_t)std::max(threads, 1), m / 4096 + 1));
  std::vector<uint64_t> bound(runs + 1);
  for (uint64_t r = 0; r <= runs; ++r) bound[r] = m * r / runs;
  par_for(runs, threads, [&](uint64_t r) { std::sort(pairs.begin() + bound[r], pairs.begin() + bound[r + 1]); });
  std::vector<P> tmp(m);
  for (uint64_t width = 1; width < runs; width *= 2) {
    const uint64_t merges = (runs + 2 * width - 1) / (2 * width);
    par_for(merges, threads, [&](uint64_t j) {
      const uint64_t a = bound[std::min(runs, 2 * width * j)], b = bound[std::min(runs, 2 * width * j + width)],
                     e = bound[std::min(runs, 2 * width * j + 2 * width)];
      std::merge(pairs.begin() + a, pairs.begin() + b, pairs.begin() + b, pairs.begin() + e, tmp.begin() + a);
    });
    pairs.swap(tmp);
  }
  uint64_t o = 0;
  if (!nulls_last)
    for (uint32_t r : nulls) out[o++] = r;
  for (const P& p : pairs) out[o++] = p.second;
  if (nulls_last)
    for (uint32_t r : nulls) out[o++] = r;
}

}  // extern "C"
