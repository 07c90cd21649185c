// gen.cpp -- seeded synthetic workloads (host side).  See include/dvg_gen.h.
#include "dvg_gen.h"

#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <new>
#include <vector>

namespace {

// splitmix64 (Steele, Lea, Flood 2014) for seeding, xoshiro256** (Blackman &
// Vigna 2018) as the stream generator.
inline uint64_t splitmix64(uint64_t& x) {
  uint64_t z = (x += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}

struct Rng {
  uint64_t s[4];
  explicit Rng(uint64_t seed) {
    uint64_t x = seed;
    for (auto& v : s) v = splitmix64(x);
  }
  static inline uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
  inline uint64_t next() {
    uint64_t r = rotl(s[1] * 5, 7) * 9;
    uint64_t t = s[1] << 17;
    s[2] ^= s[0];
    s[3] ^= s[1];
    s[1] ^= s[2];
    s[0] ^= s[3];
    s[2] ^= t;
    s[3] = rotl(s[3], 45);
    return r;
  }
  // uniform in (0, 1]
  inline double unit() { return (double((next() >> 11)) + 1.0) * (1.0 / 9007199254740992.0); }
  // uniform integer in [lo, hi]
  inline uint64_t range(uint64_t lo, uint64_t hi) {
    uint64_t span = hi - lo + 1;
    return lo + uint64_t((unsigned __int128)next() * span >> 64);
  }
  // number of failures before the first success, success probability p
  inline uint64_t geometric0(double p) {
    if (p >= 1.0) return 0;
    return uint64_t(std::floor(std::log(unit()) / std::log1p(-p)));
  }
  inline uint32_t poisson(double mean) {  // inversion by sequential search
    double l = std::exp(-mean), prod = unit();
    uint32_t k = 0;
    while (prod > l) { prod *= unit(); ++k; }
    return k;
  }
};

enum EvType : uint8_t { SNP = 0, INS = 1, DEL = 2 };
struct Event {
  uint64_t p;    // anchor: the bubble sits right after backbone base p
  uint32_t len;  // insertion / deletion length (SNP: 1)
  EvType type;
  bool sv;
};

bool valid(const dvg_graph_params* p) {
  if (!p || p->n_backbone < 2 || p->n_backbone > 0xF0000000ull) return false;
  if (p->snp_rate < 0 || p->indel_rate < 0 || p->snp_rate + p->indel_rate >= 1.0) return false;
  if (p->indel_lmin < 1 || p->indel_lmax < p->indel_lmin) return false;
  if (p->sv_frac > 0 && (p->sv_lmin < 1 || p->sv_lmax < p->sv_lmin)) return false;
  return true;
}

// Draws the bubble events in a fixed order: gap (geometric), class (uniform),
// kind (uniform), length.
std::vector<Event> draw_events(const dvg_graph_params* gp, dvg_graph_stats* st) {
  Rng rng(gp->seed);
  std::vector<Event> ev;
  const uint64_t nb = gp->n_backbone;
  const double rate = gp->snp_rate + gp->indel_rate;
  const double snp_share = rate > 0 ? gp->snp_rate / rate : 0.0;
  uint64_t next_free = 0;  // first backbone base a new anchor may use
  if (rate <= 0) return ev;
  while (true) {
    uint64_t p = next_free + rng.geometric0(rate);
    if (p >= nb) break;
    double u = rng.unit();
    double v = rng.unit();
    Event e{p, 1, SNP, false};
    if (u <= gp->sv_frac) {
      e.sv = true;
      e.type = v <= 0.5 ? INS : DEL;
      e.len = uint32_t(rng.range(gp->sv_lmin, gp->sv_lmax));
    } else if ((u - gp->sv_frac) / (1.0 - gp->sv_frac) <= snp_share) {
      e.type = SNP;
      e.len = 1;
    } else {
      e.type = v <= gp->ins_frac ? INS : DEL;
      if (gp->indel_geometric_mean > 0) {
        uint64_t l = 1 + rng.geometric0(1.0 / gp->indel_geometric_mean);
        e.len = uint32_t(std::min<uint64_t>(l, gp->indel_lmax));
      } else {
        e.len = uint32_t(rng.range(gp->indel_lmin, gp->indel_lmax));
      }
    }
    // span: SNP alters base p+1; an insertion sits between p and p+1; a
    // deletion skips bases p+1..p+len.  The bubble must close on the backbone.
    uint64_t span = e.type == SNP ? 2 : (e.type == INS ? 1 : uint64_t(e.len) + 1);
    if (p + span >= nb) { next_free = p + 1; continue; }
    ev.push_back(e);
    next_free = p + span;
  }
  if (st) {
    std::memset(st, 0, sizeof(*st));
    for (auto& e : ev) {
      if (e.sv) ++st->n_sv;
      if (e.type == SNP) { ++st->n_snp; ++st->n_alt_loci; }
      else if (e.type == INS) { ++st->n_ins; st->n_alt_loci += e.len; }
      else ++st->n_del;
    }
    st->n_loci = nb + st->n_alt_loci;
  }
  return ev;
}

// Walks the loci in topological order and reports each locus's sorted
// successor list through emit(locus, succ, nsucc).
template <class Emit>
void walk_graph(const dvg_graph_params* gp, const std::vector<Event>& ev, Emit emit) {
  const uint64_t nb = gp->n_backbone;
  uint64_t off = 0;  // alt loci numbered before backbone base p
  size_t e = 0;
  bool snp_site = false;  // backbone base p carries an SNP alt right after it
  uint64_t succ[2];
  for (uint64_t p = 0; p < nb; ++p) {
    const uint64_t L = p + off;
    const Event* here = (e < ev.size() && ev[e].p == p) ? &ev[e] : nullptr;
    if (snp_site) {
      // ref base L, alt base L+1, both lead to backbone base p+1 at L+2
      succ[0] = L + 2;
      emit(L, succ, p + 1 < nb ? 1 : 0);
      emit(L + 1, succ, p + 1 < nb ? 1 : 0);
      off += 1;
      snp_site = false;
      if (here) std::abort();  // anchors never overlap an SNP site
      continue;
    }
    if (!here) {
      succ[0] = L + 1;
      emit(L, succ, p + 1 < nb ? 1 : 0);
      continue;
    }
    ++e;
    if (here->type == SNP) {
      succ[0] = L + 1;  // ref allele at backbone p+1
      succ[1] = L + 2;  // alt allele numbered right after it
      emit(L, succ, 2);
      snp_site = true;
    } else if (here->type == INS) {
      succ[0] = L + 1;                      // first alt base
      succ[1] = L + 1 + here->len;          // backbone p+1 after the alt branch
      emit(L, succ, 2);
      for (uint32_t k = 1; k <= here->len; ++k) {
        succ[0] = L + k + 1;
        emit(L + k, succ, 1);
      }
      off += here->len;
    } else {
      succ[0] = L + 1;                      // backbone p+1
      succ[1] = L + 1 + here->len;          // backbone p+len+1
      emit(L, succ, 2);
    }
  }
}

bool alloc_matrix(dvg_host_matrix* m, uint64_t nrows, uint64_t nentries) {
  m->rowmap = (uint64_t*)std::malloc(sizeof(uint64_t) * (nrows + 1));
  m->entries = (uint32_t*)std::malloc(sizeof(uint32_t) * (nentries ? nentries : 1));
  if (!m->rowmap || !m->entries) {
    std::free(m->rowmap);
    std::free(m->entries);
    m->rowmap = nullptr;
    m->entries = nullptr;
    return false;
  }
  return true;
}

}  // namespace

extern "C" {

int dvg_gen_graph_adjacency(const dvg_graph_params* gp, dvg_host_matrix* out, dvg_graph_stats* stats) {
  if (!valid(gp) || !out) return 1;
  dvg_graph_stats st;
  std::vector<Event> ev = draw_events(gp, &st);
  if (st.n_loci >= 0xFFFFFFFEull) return 1;
  if (stats) *stats = st;
  const uint64_t n = st.n_loci;
  // at most 2 ranges per row
  if (!alloc_matrix(out, n, 4 * n)) return 2;
  out->nrows = out->ncols = uint32_t(n);
  uint64_t k = 0, nnz = 0, row = 0;
  out->rowmap[0] = 0;
  walk_graph(gp, ev, [&](uint64_t locus, const uint64_t* succ, int ns) {
    (void)locus;
    // Basic -> Range: consecutive columns merge into one range
    if (ns >= 1) {
      out->entries[k++] = uint32_t(succ[0]);
      if (ns == 2 && succ[1] == succ[0] + 1) {
        out->entries[k++] = uint32_t(succ[1]);
      } else {
        out->entries[k++] = uint32_t(succ[0]);
        if (ns == 2) {
          out->entries[k++] = uint32_t(succ[1]);
          out->entries[k++] = uint32_t(succ[1]);
        }
      }
      nnz += ns;
    }
    out->rowmap[++row] = k;
  });
  out->nentries = k;
  out->nnz = nnz;
  return row == n ? 0 : 3;
}

int dvg_gen_graph_edges(const dvg_graph_params* gp, uint64_t* n_nodes, uint64_t* n_edges, uint32_t** edges) {
  if (!valid(gp) || !n_nodes || !n_edges || !edges) return 1;
  dvg_graph_stats st;
  std::vector<Event> ev = draw_events(gp, &st);
  std::vector<uint32_t> e;
  e.reserve(2 * (st.n_loci + st.n_snp + st.n_ins + st.n_del));
  walk_graph(gp, ev, [&](uint64_t locus, const uint64_t* succ, int ns) {
    for (int i = 0; i < ns; ++i) {
      e.push_back(uint32_t(locus + 1));
      e.push_back(uint32_t(succ[i] + 1));
    }
  });
  *n_nodes = st.n_loci;
  *n_edges = e.size() / 2;
  *edges = (uint32_t*)std::malloc(sizeof(uint32_t) * (e.size() ? e.size() : 1));
  if (!*edges) return 2;
  std::memcpy(*edges, e.data(), sizeof(uint32_t) * e.size());
  return 0;
}

int dvg_gen_graph_nodes(const dvg_graph_params* gp, uint64_t* n_nodes, uint32_t** node_len, uint64_t* n_edges,
                        uint32_t** edges) {
  if (!valid(gp) || !n_nodes || !node_len || !n_edges || !edges) return 1;
  dvg_graph_stats st;
  std::vector<Event> ev = draw_events(gp, &st);
  if (st.n_loci >= 0xFFFFFFFEull) return 1;
  const uint64_t n = st.n_loci;
  // loci come in topological order, so when locus l is reached every
  // predecessor of l has been seen and its in-degree is final
  std::vector<uint8_t> indeg(n, 0);
  std::vector<uint64_t> starts;
  std::vector<uint64_t> links;  // inter-node edges as (from locus, to locus)
  bool have_prev = false;
  int prev_ns = 0;
  uint64_t prev_succ = 0;
  walk_graph(gp, ev, [&](uint64_t l, const uint64_t* succ, int ns) {
    // l opens a node unless it continues the chain of l - 1
    if (!have_prev || indeg[l] != 1 || prev_ns != 1 || prev_succ != l) starts.push_back(l);
    for (int k = 0; k < ns; ++k)
      if (indeg[succ[k]] < 255) ++indeg[succ[k]];
    for (int k = 0; k < ns; ++k) {
      const bool chain = ns == 1 && succ[k] == l + 1 && indeg[succ[k]] == 1;
      if (!chain) {
        links.push_back(l);
        links.push_back(succ[k]);
      }
    }
    have_prev = true;
    prev_ns = ns;
    prev_succ = ns ? succ[0] : 0;
  });
  const uint64_t m = starts.size();
  *n_nodes = m;
  *n_edges = links.size() / 2;
  *node_len = (uint32_t*)std::malloc(sizeof(uint32_t) * (m ? m : 1));
  *edges = (uint32_t*)std::malloc(sizeof(uint32_t) * (links.empty() ? 1 : links.size()));
  if (!*node_len || !*edges) {
    std::free(*node_len);
    std::free(*edges);
    *node_len = nullptr;
    *edges = nullptr;
    return 2;
  }
  for (uint64_t k = 0; k < m; ++k) (*node_len)[k] = uint32_t((k + 1 < m ? starts[k + 1] : n) - starts[k]);
  // node id of a locus: the number of node starts at or before it
  auto node_of = [&](uint64_t x) {
    return uint32_t(std::upper_bound(starts.begin(), starts.end(), x) - starts.begin());
  };
  for (size_t k = 0; k < links.size(); ++k) (*edges)[k] = node_of(links[k]);
  return 0;
}

int dvg_gen_banded(uint32_t n, uint32_t hw, double mean_ranges, double mean_len, uint64_t seed,
                   dvg_host_matrix* out) {
  if (!out || n == 0 || n >= 0xFFFFFFFEu || mean_ranges < 0 || mean_len < 1) return 1;
  const double pl = 1.0 / mean_len;
  std::vector<uint32_t> counts(size_t(n) + 1, 0);
  // pass 1: per-row canonical ranges into per-block buffers
  const uint32_t block = 1 << 14;
  const uint32_t nblocks = (n + block - 1) / block;
  std::vector<std::vector<uint32_t>> buf(nblocks);
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t b = 0; b < int64_t(nblocks); ++b) {
    std::vector<std::pair<uint32_t, uint32_t>> r;
    auto& out_b = buf[b];
    uint32_t r0 = uint32_t(b) * block, r1 = std::min<uint32_t>(n, r0 + block);
    for (uint32_t i = r0; i < r1; ++i) {
      uint64_t sx = seed ^ (uint64_t(i) * 0xD1B54A32D192ED03ull);
      Rng rng(splitmix64(sx));
      uint32_t k = rng.poisson(mean_ranges);
      uint64_t lo = i >= hw ? i - hw : 0;
      uint64_t hi = std::min<uint64_t>(uint64_t(i) + hw, n - 1);
      r.clear();
      for (uint32_t t = 0; t < k; ++t) {
        uint64_t s = rng.range(lo, hi);
        uint64_t len = 1 + rng.geometric0(pl);
        uint64_t f = std::min<uint64_t>(s + len - 1, hi);
        r.emplace_back(uint32_t(s), uint32_t(f));
      }
      std::sort(r.begin(), r.end());
      uint32_t cnt = 0;
      for (size_t t = 0; t < r.size();) {
        uint32_t s = r[t].first, f = r[t].second;
        size_t u = t + 1;
        while (u < r.size() && uint64_t(r[u].first) <= uint64_t(f) + 1) { f = std::max(f, r[u].second); ++u; }
        out_b.push_back(s);
        out_b.push_back(f);
        cnt += 2;
        t = u;
      }
      counts[i + 1] = cnt;
    }
  }
  uint64_t total = 0;
  for (auto& v : buf) total += v.size();
  if (!alloc_matrix(out, n, total)) return 2;
  out->nrows = out->ncols = n;
  out->rowmap[0] = 0;
  for (uint32_t i = 0; i < n; ++i) out->rowmap[i + 1] = out->rowmap[i] + counts[i + 1];
  uint64_t pos = 0;
  for (auto& v : buf) {
    if (!v.empty()) std::memcpy(out->entries + pos, v.data(), 4 * v.size());
    pos += v.size();
  }
  uint64_t nnz = 0;
#pragma omp parallel for reduction(+ : nnz)
  for (int64_t t = 0; t < int64_t(total / 2); ++t) nnz += uint64_t(out->entries[2 * t + 1]) - out->entries[2 * t] + 1;
  out->nentries = total;
  out->nnz = nnz;
  return 0;
}

int dvg_gen_random(uint32_t n, uint64_t nnz, uint64_t seed, dvg_host_matrix* out) {
  if (!out || n < 2 || nnz == 0 || nnz > uint64_t(n) * n) return 1;
  Rng rng(seed);
  std::vector<uint64_t> rowcnt(n, 0);
  for (uint64_t t = 0; t < nnz; ++t) {
    uint64_t r = rng.range(0, n - 1);
    while (rowcnt[r] >= n) r = (r + 1) % n;
    ++rowcnt[r];
  }
  std::vector<uint64_t> rowmap(size_t(n) + 1, 0);
  std::vector<uint32_t> ent;
  std::vector<uint32_t> cols;
  for (uint32_t i = 0; i < n; ++i) {
    // Floyd's sampling of rowcnt[i] distinct columns
    cols.clear();
    uint64_t k = rowcnt[i];
    if (k * 2 > n) {
      for (uint32_t c = 0; c < n; ++c) cols.push_back(c);
      for (uint64_t t = 0; t + 1 < n; ++t) std::swap(cols[t], cols[rng.range(t, n - 1)]);
      cols.resize(k);
    } else {
      std::vector<uint32_t> pick;
      for (uint64_t j = n - k; j < n; ++j) {
        uint32_t t = uint32_t(rng.range(0, j));
        if (std::find(pick.begin(), pick.end(), t) != pick.end()) pick.push_back(uint32_t(j));
        else pick.push_back(t);
      }
      cols = pick;
    }
    std::sort(cols.begin(), cols.end());
    bool pending = false;
    uint32_t pend = 0;
    for (uint32_t c : cols) {
      if (pending && c == pend + 1) { ++pend; continue; }
      if (pending) ent.push_back(pend);
      ent.push_back(c);
      pend = c;
      pending = true;
    }
    if (pending) ent.push_back(pend);
    rowmap[i + 1] = ent.size();
  }
  if (!alloc_matrix(out, n, ent.size())) return 2;
  out->nrows = out->ncols = n;
  std::memcpy(out->rowmap, rowmap.data(), sizeof(uint64_t) * rowmap.size());
  if (!ent.empty()) std::memcpy(out->entries, ent.data(), 4 * ent.size());
  out->nentries = ent.size();
  out->nnz = nnz;
  return 0;
}

int dvg_gen_pairs(const dvg_host_matrix* adj, uint64_t npairs, double in_range_frac, uint32_t dmin,
                  uint32_t dmax, uint64_t seed, uint32_t* pairs) {
  if (!adj || !pairs || adj->nrows == 0 || dmin > dmax) return 1;
  const uint32_t n = adj->nrows;
  const uint64_t chunk = 1 << 16;
  const uint64_t nchunks = (npairs + chunk - 1) / chunk;
#pragma omp parallel for schedule(dynamic, 1)
  for (int64_t c = 0; c < int64_t(nchunks); ++c) {
    uint64_t sx = seed ^ (uint64_t(c) * 0x9E3779B97F4A7C15ull);
    Rng rng(splitmix64(sx));
    uint64_t q1 = std::min<uint64_t>(npairs, uint64_t(c + 1) * chunk);
    for (uint64_t q = uint64_t(c) * chunk; q < q1; ++q) {
      uint32_t i = uint32_t(rng.range(0, n - 1));
      uint32_t j;
      if (rng.unit() <= in_range_frac) {
        uint32_t d = uint32_t(rng.range(dmin, dmax));
        j = i;
        for (uint32_t t = 0; t < d; ++t) {
          uint64_t b = adj->rowmap[j], e = adj->rowmap[j + 1];
          if (b == e) break;
          j = adj->entries[b];
        }
      } else {
        j = uint32_t(rng.range(0, n - 1));
      }
      pairs[2 * q] = i;
      pairs[2 * q + 1] = j;
    }
  }
  return 0;
}

void dvg_gen_free(dvg_host_matrix* m) {
  if (!m) return;
  std::free(m->rowmap);
  std::free(m->entries);
  m->rowmap = nullptr;
  m->entries = nullptr;
}

void dvg_gen_free_ptr(void* p) { std::free(p); }

}  // extern "C"
