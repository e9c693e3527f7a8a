// Shared pieces of the native host mesh builders (mesh2d.cpp, geom3d.cpp): the table
// container returned through the C ABI and the CSR / SELL-32 / ordering helpers.  Each
// helper reproduces the numpy operation it replaces (stable orders, sorted unique unions).
#pragma once
#include <algorithm>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <numeric>
#include <string>
#include <thread>
#include <vector>

namespace mbh {

using i32 = int32_t;
using i64 = int64_t;

// An allocator whose value-less construct() leaves scalars uninitialised: a vector sized
// with it is not zero-filled, so the (parallel) loop that fills it is the first to touch
// its pages.
template <class T>
struct NoInit : std::allocator<T> {
  template <class U>
  struct rebind {
    using other = NoInit<U>;
  };
  NoInit() = default;
  template <class U>
  NoInit(const NoInit<U> &) {}
  template <class U>
  void construct(U *p) noexcept {
    ::new (static_cast<void *>(p)) U;
  }
  template <class U, class... A>
  void construct(U *p, A &&...a) {
    ::new (static_cast<void *>(p)) U(std::forward<A>(a)...);
  }
};
template <class T>
using uvec = std::vector<T, NoInit<T>>;

struct Table {
  std::string name;
  char dtype;  // 'i' int32, 'l' int64, 'd' float64, 'f' float32, 'b' uint8
  std::vector<i64> shape;
  std::shared_ptr<void> owner;  // the storage of the table's bytes
  const void *data = nullptr;
  size_t nbytes = 0;
};

struct Result {
  std::vector<Table> tables;
  std::string error;
  // the table takes over v's storage (no copy)
  template <class T, class A>
  void add(const std::string &name, char dt, std::vector<i64> shape, std::vector<T, A> &&v) {
    auto held = std::make_shared<std::vector<T, A>>(std::move(v));
    Table t;
    t.name = name;
    t.dtype = dt;
    t.shape = std::move(shape);
    t.data = held->data();
    t.nbytes = held->size() * sizeof(T);
    t.owner = std::move(held);
    tables.push_back(std::move(t));
  }
  // a table of a vector that the builder still uses: copied
  template <class T, class A>
  void add(const std::string &name, char dt, std::vector<i64> shape, const std::vector<T, A> &v) {
    add(name, dt, std::move(shape), std::vector<T, A>(v));
  }
};

// Host threads for n independent items: up to 16 (or MANAPY_B200_HOST_THREADS, for a process
// that shares the cores with others), one below min_n items.
inline i64 pool_size(i64 n, i64 min_n) {
  i64 cap = (i64)std::max(1u, std::min(16u, std::thread::hardware_concurrency()));
  if (const char *env = std::getenv("MANAPY_B200_HOST_THREADS")) {
    const long v = std::strtol(env, nullptr, 10);
    if (v > 0) cap = v;
  }
  return n >= min_n ? std::max<i64>(1, std::min<i64>(cap, n)) : 1;
}

// fn(t, i0, i1) for t < nt over the contiguous ranges [n t / nt, n (t+1) / nt), each on its
// own thread (range 0 on the calling one).  fn writes only what its range owns, so the
// result does not depend on nt.
template <class F>
inline void run_ranges(i64 nt, i64 n, F &&fn) {
  if (nt <= 1) {
    fn((i64)0, (i64)0, n);
    return;
  }
  std::vector<std::thread> pool;
  pool.reserve(nt - 1);
  for (i64 t = 1; t < nt; ++t) pool.emplace_back([&, t] { fn(t, n * t / nt, n * (t + 1) / nt); });
  fn((i64)0, (i64)0, n / nt);
  for (auto &th : pool) th.join();
}

// fn(i) for every i in [0, n), split over host threads when n is large.
template <class F>
inline void parallel_for(i64 n, F &&fn) {
  run_ranges(pool_size(n, (i64)1 << 15), n, [&](i64, i64 i0, i64 i1) {
    for (i64 i = i0; i < i1; ++i) fn(i);
  });
}

// out = the elements of `in` (or 0, 1, ... when in is null) in stable order of digit[e] in
// [0, n): a counting sort.  Large inputs are counted and scattered by host threads, each over
// a contiguous range of the input, from per-thread offsets (digit-major, then thread), so
// the order is the serial one.
inline void stable_by_digit(const std::vector<i64> &digit, const std::vector<i64> *in, i64 m, i64 n,
                            std::vector<i64> &out) {
  out.resize(m);
  auto elem = [&](i64 e) { return in ? (*in)[e] : e; };
  const i64 nt = std::min<i64>(pool_size(m, (i64)1 << 18), std::max<i64>(1, m / std::max<i64>(n, 1)));
  if (nt <= 1) {
    std::vector<i64> pos(n + 1, 0);
    for (i64 e = 0; e < m; ++e) pos[digit[elem(e)] + 1]++;
    for (i64 d = 0; d < n; ++d) pos[d + 1] += pos[d];
    for (i64 e = 0; e < m; ++e) {
      const i64 x = elem(e);
      out[pos[digit[x]]++] = x;
    }
    return;
  }
  std::vector<i64> cnt(nt * n, 0);  // cnt[t * n + d]
  run_ranges(nt, m, [&](i64 t, i64 e0, i64 e1) {
    i64 *c = &cnt[t * n];
    for (i64 e = e0; e < e1; ++e) c[digit[elem(e)]]++;
  });
  i64 run = 0;
  for (i64 d = 0; d < n; ++d)
    for (i64 t = 0; t < nt; ++t) {
      const i64 c = cnt[t * n + d];
      cnt[t * n + d] = run;
      run += c;
    }
  run_ranges(nt, m, [&](i64 t, i64 e0, i64 e1) {
    i64 *c = &cnt[t * n];
    for (i64 e = e0; e < e1; ++e) {
      const i64 x = elem(e);
      out[c[digit[x]]++] = x;
    }
  });
}

// Stable argsort of integer keys in [0, n): a counting sort (equal keys keep their order).
inline std::vector<i64> counting_argsort(const std::vector<i64> &key, i64 n) {
  std::vector<i64> o;
  stable_by_digit(key, nullptr, (i64)key.size(), n, o);
  return o;
}

// CSR rows taken in `rows` order with values mapped through vinv, each row's entry order
// kept; src (optional) gets each new entry's position in the old table.
inline void relabel_csr(const std::vector<i64> &ptr, const std::vector<i64> &idx, const std::vector<i64> &rows,
                        const std::vector<i64> &vinv, std::vector<i64> &optr, std::vector<i64> &oidx,
                        std::vector<i64> *src) {
  const i64 n = (i64)rows.size();
  optr.assign(n + 1, 0);
  for (i64 r = 0; r < n; ++r) optr[r + 1] = optr[r] + (ptr[rows[r] + 1] - ptr[rows[r]]);
  oidx.resize(optr[n]);
  if (src) src->resize(optr[n]);
  parallel_for(n, [&](i64 r) {
    i64 e = optr[r];
    for (i64 a = ptr[rows[r]]; a < ptr[rows[r] + 1]; ++a, ++e) {
      oidx[e] = vinv[idx[a]];
      if (src) (*src)[e] = a;
    }
  });
}

// CSR from (key, value) pairs grouped by key in [0, n), values kept in input order (a
// stable counting sort, as numpy's stable argsort of the keys)
inline void group_csr(const std::vector<i64> &key, const std::vector<i64> &val, i64 n, std::vector<i64> &ptr,
               std::vector<i64> &idx) {
  ptr.assign(n + 1, 0);
  for (i64 k : key) ptr[k + 1]++;
  for (i64 i = 0; i < n; ++i) ptr[i + 1] += ptr[i];
  std::vector<i64> order;
  stable_by_digit(key, nullptr, (i64)key.size(), n, order);
  idx.resize(key.size());
  parallel_for((i64)key.size(), [&](i64 e) { idx[e] = val[order[e]]; });
}

// for each row r: sorted unique union of the lists of its items (CSR), optionally without r.
// Item lists that are ascending (node -> cell and node -> face lists are) are merged; any
// other row is gathered and sorted.  Large tables are split into row ranges handled by
// separate threads; each range's output is concatenated in row order (same result).
inline void ragged_union(i64 nrows, const std::vector<i64> &row_items_ptr, const std::vector<i64> &row_items,
                         const std::vector<i64> &item_ptr, const std::vector<i64> &item_vals, bool exclude_self,
                         std::vector<i64> &ptr, std::vector<i64> &idx) {
  const i64 nitems = (i64)item_ptr.size() - 1;
  std::vector<char> ascending(nitems, 1);
  for (i64 it = 0; it < nitems; ++it)
    for (i64 b = item_ptr[it] + 1; b < item_ptr[it + 1]; ++b)
      if (item_vals[b] < item_vals[b - 1]) {
        ascending[it] = 0;
        break;
      }
  // rows [r0, r1): per-row counts into cnt[r], values appended to out
  auto rows = [&](i64 r0, i64 r1, i64 *cnt, std::vector<i64> &out) {
    std::vector<i64> buf, pos, end;
    for (i64 r = r0; r < r1; ++r) {
      const size_t before = out.size();
      bool merge = true;
      for (i64 a = row_items_ptr[r]; a < row_items_ptr[r + 1]; ++a) merge = merge && ascending[row_items[a]];
      bool have = false;
      i64 last = 0;
      auto emit = [&](i64 v) {
        if (have && v == last) return;
        have = true;
        last = v;
        if (exclude_self && v == r) return;
        out.push_back(v);
      };
      if (merge) {
        pos.clear();
        end.clear();
        for (i64 a = row_items_ptr[r]; a < row_items_ptr[r + 1]; ++a) {
          const i64 it = row_items[a];
          if (item_ptr[it] < item_ptr[it + 1]) {
            pos.push_back(item_ptr[it]);
            end.push_back(item_ptr[it + 1]);
          }
        }
        const size_t k = pos.size();
        for (;;) {
          int best = -1;
          i64 v = 0;
          for (size_t h = 0; h < k; ++h)
            if (pos[h] < end[h] && (best < 0 || item_vals[pos[h]] < v)) {
              best = (int)h;
              v = item_vals[pos[h]];
            }
          if (best < 0) break;
          ++pos[best];
          emit(v);
        }
      } else {
        buf.clear();
        for (i64 a = row_items_ptr[r]; a < row_items_ptr[r + 1]; ++a) {
          const i64 it = row_items[a];
          for (i64 b = item_ptr[it]; b < item_ptr[it + 1]; ++b) buf.push_back(item_vals[b]);
        }
        std::sort(buf.begin(), buf.end());
        for (i64 v : buf) emit(v);
      }
      cnt[r] = (i64)(out.size() - before);
    }
  };
  std::vector<i64> cnt(nrows);
  const i64 nthreads = pool_size(nrows, (i64)1 << 16);
  std::vector<std::vector<i64>> parts(nthreads);
  run_ranges(nthreads, nrows, [&](i64 t, i64 r0, i64 r1) { rows(r0, r1, cnt.data(), parts[t]); });
  ptr.assign(nrows + 1, 0);
  for (i64 r = 0; r < nrows; ++r) ptr[r + 1] = ptr[r] + cnt[r];
  idx.clear();
  idx.reserve(ptr[nrows]);
  for (auto &p : parts) idx.insert(idx.end(), p.begin(), p.end());
}

// SELL-32 of a CSR table (rows in warps of 32, entry k of the 32 rows contiguous);
// padding: -1, or (fill_first) the row's first entry with value 0
inline void sell32(const std::vector<i64> &ptr, const std::vector<i64> &idx, const std::vector<double> *vals,
            bool fill_first, std::vector<i32> &gptr, std::vector<i32> &out, std::vector<double> &outv) {
  const i64 n = (i64)ptr.size() - 1;
  const i64 ng = (n + 31) / 32;
  gptr.assign(ng + 1, 0);
  std::vector<i64> g64(ng + 1, 0);
  for (i64 g = 0; g < ng; ++g) {
    i64 len = 0;
    for (i64 r = 32 * g; r < std::min(n, 32 * g + 32); ++r) len = std::max(len, ptr[r + 1] - ptr[r]);
    g64[g + 1] = g64[g] + 32 * len;
  }
  out.assign(g64[ng], -1);
  outv.assign(vals ? g64[ng] : 0, 0.0);
  parallel_for(ng, [&](i64 g) {
    const i64 len = (g64[g + 1] - g64[g]) / 32;
    for (i64 l = 0; l < 32; ++l) {
      const i64 r = 32 * g + l;
      const i64 cnt = r < n ? ptr[r + 1] - ptr[r] : 0;
      const i64 first = (r < n && cnt > 0) ? idx[ptr[r]] : 0;
      for (i64 k = 0; k < len; ++k) {
        const i64 d = g64[g] + 32 * k + l;
        if (k < cnt) {
          out[d] = (i32)idx[ptr[r] + k];
          if (vals) outv[d] = (*vals)[ptr[r] + k];
        } else if (fill_first) {
          out[d] = (i32)first;
        }
      }
    }
  });
  for (i64 g = 0; g <= ng; ++g) gptr[g] = (i32)g64[g];
}

// SELL-32 whose slots are shared across each warp's 32 rows: a value that several rows of
// the warp hold is placed, where their free slots allow, in one slot for all of them, so
// that a warp-wide gather of slot k touches few distinct addresses.  Per warp: every
// distinct value with the mask of rows holding it, taken in order of decreasing row count
// (then ascending value); each goes to the slot with the most of its remaining rows free
// (the first such slot), and what stays unplaced goes on the same way.  A row keeps each
// of its entries exactly once; the slot count is the warp's longest row + slack (a row
// with fewer entries than slots always has a free slot).  Empty slots hold -1.  The order
// of a row's entries is the slot order (not the CSR order).  Warps in parallel threads.
inline void sell32_aligned(const std::vector<i64> &ptr, const std::vector<i64> &idx, int slack,
                           std::vector<i32> &gptr, std::vector<i32> &out) {
  const i64 n = (i64)ptr.size() - 1;
  const i64 ng = (n + 31) / 32;
  std::vector<i64> g64(ng + 1, 0);
  for (i64 g = 0; g < ng; ++g) {
    i64 len = 0;
    for (i64 r = 32 * g; r < std::min(n, 32 * g + 32); ++r) len = std::max(len, ptr[r + 1] - ptr[r]);
    g64[g + 1] = g64[g] + 32 * (len + (len ? slack : 0));
  }
  out.resize(g64[ng]);
  auto warps = [&](i64 g0, i64 g1) {
    std::vector<std::pair<i64, int>> pairs;        // (value, row in warp)
    std::vector<std::pair<i64, uint32_t>> els;     // (value, rows mask)
    std::vector<std::pair<std::pair<i64, int>, uint32_t>> keyed;
    std::vector<uint32_t> occ;
    std::fill(out.begin() + g64[g0], out.begin() + g64[g1], -1);   // this range's slots, empty
    for (i64 g = g0; g < g1; ++g) {
      const i64 L = (g64[g + 1] - g64[g]) / 32;
      if (!L) continue;
      pairs.clear();
      for (i64 r = 32 * g; r < std::min(n, 32 * g + 32); ++r)
        for (i64 e = ptr[r]; e < ptr[r + 1]; ++e) pairs.emplace_back(idx[e], (int)(r - 32 * g));
      std::sort(pairs.begin(), pairs.end());
      // a value repeated within one row counts as distinct values (its k-th copies grouped)
      els.clear();
      keyed.clear();
      for (size_t a = 0; a < pairs.size();) {
        size_t b = a;
        while (b < pairs.size() && pairs[b].first == pairs[a].first) ++b;
        // rows of this value, with the copy number of each occurrence
        int copy = 0;
        for (size_t c = a; c < b; ++c) {
          copy = (c > a && pairs[c].second == pairs[c - 1].second) ? copy + 1 : 0;
          bool merged = false;
          for (auto &kv : keyed)
            if (kv.first.first == pairs[c].first && kv.first.second == copy && !(kv.second >> pairs[c].second & 1u)) {
              kv.second |= 1u << pairs[c].second;
              merged = true;
              break;
            }
          if (!merged) keyed.push_back({{pairs[c].first, copy}, 1u << pairs[c].second});
        }
        for (auto &kv : keyed) els.emplace_back(kv.first.first, kv.second);
        keyed.clear();
        a = b;
      }
      std::stable_sort(els.begin(), els.end(), [](const std::pair<i64, uint32_t> &x, const std::pair<i64, uint32_t> &y) {
        const int cx = __builtin_popcount(x.second), cy = __builtin_popcount(y.second);
        return cx != cy ? cx > cy : x.first < y.first;
      });
      occ.assign(L, 0u);
      for (const auto &el : els) {
        uint32_t rem = el.second;
        while (rem) {
          i64 best = -1;
          int bc = 0;
          for (i64 k = 0; k < L; ++k) {
            const uint32_t f = rem & ~occ[k];
            const int c = __builtin_popcount(f);
            if (c > bc) {
              bc = c;
              best = k;
              if (f == rem) break;
            }
          }
          const uint32_t f = rem & ~occ[best];
          occ[best] |= f;
          for (uint32_t m = f; m; m &= m - 1) out[g64[g] + 32 * best + __builtin_ctz(m)] = (i32)el.first;
          rem &= ~f;
        }
      }
    }
  };
  run_ranges(pool_size(ng, 2048), ng, [&](i64, i64 g0, i64 g1) { warps(g0, g1); });
  gptr.assign(ng + 1, 0);
  for (i64 g = 0; g <= ng; ++g) gptr[g] = (i32)g64[g];
}

inline uint64_t part1by1(uint64_t v) {
  v &= 0xFFFFFFFFull;
  v = (v | (v << 16)) & 0x0000FFFF0000FFFFull;
  v = (v | (v << 8)) & 0x00FF00FF00FF00FFull;
  v = (v | (v << 4)) & 0x0F0F0F0F0F0F0F0Full;
  v = (v | (v << 2)) & 0x3333333333333333ull;
  v = (v | (v << 1)) & 0x5555555555555555ull;
  return v;
}

// Stable argsort of unsigned keys: LSD radix passes of 11 bits up to the largest key's top
// bit (each pass a stable counting sort), the same order as a stable comparison sort.
inline std::vector<i64> radix_argsort(const std::vector<uint64_t> &key) {
  const i64 n = (i64)key.size();
  uint64_t top = 0;
  for (uint64_t k : key) top |= k;
  int bits = 0;
  while (bits < 64 && (top >> bits)) ++bits;
  std::vector<i64> o(n), tmp(n);
  std::iota(o.begin(), o.end(), 0);
  constexpr int D = 11;
  std::vector<i64> cnt((1 << D) + 1);
  for (int sh = 0; sh < bits; sh += D) {
    std::fill(cnt.begin(), cnt.end(), 0);
    for (i64 e = 0; e < n; ++e) cnt[((key[e] >> sh) & ((1u << D) - 1)) + 1]++;
    for (int d = 0; d < (1 << D); ++d) cnt[d + 1] += cnt[d];
    for (i64 e = 0; e < n; ++e) {
      const i64 x = o[e];
      tmp[cnt[(key[x] >> sh) & ((1u << D) - 1)]++] = x;
    }
    o.swap(tmp);
  }
  return o;
}

template <class K>
inline std::vector<i64> stable_argsort(const std::vector<K> &key) {
  std::vector<i64> o(key.size());
  std::iota(o.begin(), o.end(), 0);
  std::stable_sort(o.begin(), o.end(), [&](i64 a, i64 b) { return key[a] < key[b]; });
  return o;
}


}  // namespace mbh
