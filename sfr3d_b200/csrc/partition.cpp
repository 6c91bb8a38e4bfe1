// Row partition of one global CSRD system into the per-rank layouts and
// interface maps of the reference's MPI path.
//
// The reference gets its partition from a mesh pre-partitioner and lets
// dataStruct build each rank's matrix (Datastruct.c:129-190 for symmetric
// CSRD: the strict lower square part plus a rectangular CSR of the ghost
// columns; the unsymmetric branch keeps full rows whose ghost columns are
// numbered after the owned ones).  The interface that comunicateNeq uses
// (ParallelMpi.c:3346-3418) lists, per neighbour, the owned values sent and
// the ghost values received.  This file builds the same from a global
// system: each rank numbers its rows in global order, then its ghosts
// grouped by owning rank and, within a rank, by global number ("numeradas
// primeiro por vizinho e depois por numeracao global", ParallelMpi.c:3341);
// a rank sends a neighbour its rows that the neighbour references, in the
// neighbour's ghost order, so both sides agree without talking.
#include <algorithm>
#include <cstdint>
#include <cstring>
#include <new>
#include <string>
#include <vector>

#include "internal.h"

namespace sfr {
void set_last_error(const char *msg);
}

struct sfr_part {
  int32_t neq = 0, nparts = 0, unsym = 0;
  // full off-diagonal adjacency of the global matrix: column and index of
  // the value in the global al, per row in stored order (unsym) or lower
  // entries then mirrored upper ones (sym)
  std::vector<int64_t> ptr;
  std::vector<int32_t> col, src;
  std::vector<int32_t> owner;  // rank of each row
  std::vector<int32_t> lidx;   // local index of each row on its owner
  struct Rank {
    std::vector<int32_t> rows;   // owned rows, ascending
    std::vector<int32_t> ghosts; // ghost rows in local order
    std::vector<int32_t> viz;    // neighbour ranks, ascending
    std::vector<int32_t> ia_rcv, ia_snd;  // per neighbour, into xb
    std::vector<int32_t> fmap;            // nRcvs + nSends local equations
    std::vector<int32_t> ia, ja, jsrc;
    int32_t nad = 0, nadr = 0;
  };
  std::vector<Rank> ranks;
};

namespace {

int bad(const char *msg) {
  sfr::set_last_error(msg);
  return SFR_BAD_INPUT;
}

// sorts the entries [b, e) of (ja, src) by column
void sort_row(std::vector<int32_t> &ja, std::vector<int32_t> &src, size_t b, size_t e) {
  std::vector<std::pair<int32_t, int32_t>> t;
  t.reserve(e - b);
  for (size_t k = b; k < e; ++k) t.emplace_back(ja[k], src[k]);
  std::stable_sort(t.begin(), t.end(),
                   [](const auto &x, const auto &y) { return x.first < y.first; });
  for (size_t k = b; k < e; ++k) {
    ja[k] = t[k - b].first;
    src[k] = t[k - b].second;
  }
}

}  // namespace

extern "C" {

int sfr_part_create(int32_t neq, const int32_t *ia, const int32_t *ja, int32_t unsym,
                    int32_t nparts, const int32_t *part, sfr_part **out) {
  if (!out) return bad("out is NULL");
  *out = nullptr;
  if (neq <= 0 || !ia || nparts <= 0 || nparts > 32767)
    return bad("neq and nparts must be positive (nparts < 32768) and ia non-NULL");
  const int32_t base = ia[0];
  if (base < 0) return bad("ia[0] negative");
  for (int32_t i = 0; i < neq; ++i)
    if (ia[i + 1] < ia[i]) return bad("ia not monotone");
  const int64_t cnt = static_cast<int64_t>(ia[neq]) - base;
  if (cnt > 0 && !ja) return bad("ja is NULL");
  for (int64_t k = 0; k < cnt; ++k)
    if (ja[base + k] < 0 || ja[base + k] >= neq) return bad("ja out of range");
  if (!unsym)
    for (int32_t i = 0; i < neq; ++i)
      for (int32_t k = ia[i]; k < ia[i + 1]; ++k)
        if (ja[k] >= i) return bad("entry not strictly lower in the symmetric storage");
  if (part)
    for (int32_t i = 0; i < neq; ++i)
      if (part[i] < 0 || part[i] >= nparts) return bad("part[i] out of range");

  sfr_part *p = new (std::nothrow) sfr_part;
  if (!p) return bad("out of host memory");
  p->neq = neq;
  p->nparts = nparts;
  p->unsym = unsym ? 1 : 0;
  // full adjacency
  p->ptr.assign(static_cast<size_t>(neq) + 1, 0);
  if (unsym) {
    p->col.resize(cnt);
    p->src.resize(cnt);
    for (int32_t i = 0; i < neq; ++i) {
      p->ptr[i + 1] = ia[i + 1] - base;
      for (int32_t k = ia[i]; k < ia[i + 1]; ++k) {
        p->col[k - base] = ja[k];
        p->src[k - base] = k - base;
      }
    }
  } else {
    std::vector<int64_t> up(static_cast<size_t>(neq) + 1, 0);
    for (int64_t k = 0; k < cnt; ++k) ++up[ja[base + k] + 1];
    for (int32_t i = 0; i < neq; ++i)
      p->ptr[i + 1] = p->ptr[i] + (ia[i + 1] - ia[i]) + up[i + 1];
    std::vector<int64_t> fill(p->ptr.begin(), p->ptr.end() - 1);
    p->col.resize(2 * cnt);
    p->src.resize(2 * cnt);
    for (int32_t i = 0; i < neq; ++i)
      for (int32_t k = ia[i]; k < ia[i + 1]; ++k) {
        const int64_t q = fill[i]++;
        p->col[q] = ja[k];
        p->src[q] = k - base;
      }
    for (int32_t i = 0; i < neq; ++i)
      for (int32_t k = ia[i]; k < ia[i + 1]; ++k) {
        const int64_t q = fill[ja[k]]++;
        p->col[q] = i;
        p->src[q] = k - base;
      }
  }
  // owners: given, or contiguous blocks with about equal (1 + row entries)
  p->owner.resize(neq);
  if (part) {
    std::copy(part, part + neq, p->owner.begin());
  } else {
    const int64_t total = neq + static_cast<int64_t>(p->ptr[neq]);
    int64_t acc = 0;
    for (int32_t i = 0; i < neq; ++i) {
      const int64_t w = 1 + (p->ptr[i + 1] - p->ptr[i]);
      // the rank whose share contains the row's midpoint
      const int64_t mid2 = 2 * acc + w;
      p->owner[i] = static_cast<int32_t>(std::min<int64_t>(
          nparts - 1, (mid2 * nparts) / (2 * total)));
      acc += w;
    }
  }
  p->ranks.resize(nparts);
  p->lidx.resize(neq);
  for (int32_t i = 0; i < neq; ++i) {
    auto &R = p->ranks[p->owner[i]];
    p->lidx[i] = static_cast<int32_t>(R.rows.size());
    R.rows.push_back(i);
  }
  // ghosts and receive lists
  std::vector<int32_t> mark(neq, -1);
  for (int32_t r = 0; r < nparts; ++r) {
    auto &R = p->ranks[r];
    std::vector<std::pair<int32_t, int32_t>> gh;  // (owner, global)
    for (int32_t i : R.rows)
      for (int64_t q = p->ptr[i]; q < p->ptr[i + 1]; ++q) {
        const int32_t c = p->col[q];
        if (p->owner[c] != r && mark[c] != r) {
          mark[c] = r;
          gh.emplace_back(p->owner[c], c);
        }
      }
    std::sort(gh.begin(), gh.end());
    R.ghosts.reserve(gh.size());
    for (auto &g : gh) R.ghosts.push_back(g.second);
  }
  // neighbours: ranks this one receives from or sends to
  std::vector<std::vector<std::vector<int32_t>>> sends(nparts);  // sends[r][q]: rows r sends q
  for (int32_t q = 0; q < nparts; ++q)
    for (int32_t g : p->ranks[q].ghosts) {
      auto &s = sends[p->owner[g]];
      if (s.empty()) s.resize(nparts);
      s[q].push_back(g);
    }
  for (int32_t r = 0; r < nparts; ++r) {
    auto &R = p->ranks[r];
    const int32_t nown = static_cast<int32_t>(R.rows.size());
    std::vector<int32_t> from(nparts, 0);
    for (int32_t g : R.ghosts) ++from[p->owner[g]];
    for (int32_t q = 0; q < nparts; ++q) {
      const bool snd = !sends[r].empty() && !sends[r][q].empty();
      if (q != r && (from[q] > 0 || snd)) R.viz.push_back(q);
    }
    const int32_t nrcv = static_cast<int32_t>(R.ghosts.size());
    R.ia_rcv.assign(1, 0);
    for (int32_t q : R.viz) R.ia_rcv.push_back(R.ia_rcv.back() + from[q]);
    R.fmap.resize(nrcv);
    for (int32_t k = 0; k < nrcv; ++k) R.fmap[k] = nown + k;
    R.ia_snd.assign(1, nrcv);
    for (int32_t q : R.viz) {
      const auto *lst = sends[r].empty() ? nullptr : &sends[r][q];
      if (lst)
        for (int32_t g : *lst) R.fmap.push_back(p->lidx[g]);
      R.ia_snd.push_back(static_cast<int32_t>(R.fmap.size()));
    }
  }
  // local matrices
  for (int32_t r = 0; r < nparts; ++r) {
    auto &R = p->ranks[r];
    const int32_t nown = static_cast<int32_t>(R.rows.size());
    std::vector<int32_t> gl(R.ghosts.size());
    for (size_t k = 0; k < R.ghosts.size(); ++k) mark[R.ghosts[k]] = -2 - static_cast<int32_t>(k);
    auto local_col = [&](int32_t c) {
      return p->owner[c] == r ? p->lidx[c] : nown + (-2 - mark[c]);
    };
    if (unsym) {
      R.ia.assign(1, 0);
      for (int32_t i : R.rows) {
        const size_t b = R.ja.size();
        for (int64_t q = p->ptr[i]; q < p->ptr[i + 1]; ++q) {
          R.ja.push_back(local_col(p->col[q]));
          R.jsrc.push_back(p->src[q]);
        }
        sort_row(R.ja, R.jsrc, b, R.ja.size());
        R.ia.push_back(static_cast<int32_t>(R.ja.size()));
      }
      R.nad = static_cast<int32_t>(R.ja.size());
      R.nadr = 0;
    } else {
      // square strict-lower part, then the ghost columns of the full rows
      R.ia.assign(1, 0);
      for (int32_t li = 0; li < nown; ++li) {
        const int32_t i = R.rows[li];
        const size_t b = R.ja.size();
        for (int64_t q = p->ptr[i]; q < p->ptr[i + 1]; ++q) {
          const int32_t c = p->col[q];
          if (p->owner[c] == r && p->lidx[c] < li) {
            R.ja.push_back(p->lidx[c]);
            R.jsrc.push_back(p->src[q]);
          }
        }
        sort_row(R.ja, R.jsrc, b, R.ja.size());
        R.ia.push_back(static_cast<int32_t>(R.ja.size()));
      }
      R.nad = static_cast<int32_t>(R.ja.size());
      R.ia.push_back(0);
      for (int32_t li = 0; li < nown; ++li) {
        const int32_t i = R.rows[li];
        const size_t b = R.ja.size();
        for (int64_t q = p->ptr[i]; q < p->ptr[i + 1]; ++q) {
          const int32_t c = p->col[q];
          if (p->owner[c] != r) {
            R.ja.push_back(local_col(c));
            R.jsrc.push_back(p->src[q]);
          }
        }
        sort_row(R.ja, R.jsrc, b, R.ja.size());
        R.ia.push_back(static_cast<int32_t>(R.ja.size()) - R.nad);
      }
      R.nadr = static_cast<int32_t>(R.ja.size()) - R.nad;
    }
    for (int32_t g : R.ghosts) mark[g] = -1;
  }
  *out = p;
  return SFR_OK;
}

int sfr_part_sizes_of(const sfr_part *p, int32_t rank, sfr_part_sizes *sz) {
  if (!p || !sz || rank < 0 || rank >= p->nparts) return bad("bad partition, rank or sizes");
  const auto &R = p->ranks[rank];
  sz->nEqNov = static_cast<int32_t>(R.rows.size());
  sz->nEq = sz->nEqNov + static_cast<int32_t>(R.ghosts.size());
  sz->nAd = R.nad;
  sz->nAdR = R.nadr;
  sz->nRcvs = static_cast<int32_t>(R.ghosts.size());
  sz->nSends = static_cast<int32_t>(R.fmap.size()) - sz->nRcvs;
  sz->nVizPart = static_cast<int32_t>(R.viz.size());
  sz->ia_len = static_cast<int32_t>(R.ia.size());
  return SFR_OK;
}

int sfr_part_fill(const sfr_part *p, int32_t rank, int32_t *ia, int32_t *ja, int32_t *src,
                  int32_t *l2g, int32_t *iaSends, int32_t *iaRcvs, int32_t *fMap,
                  int16_t *vizPart) {
  if (!p || rank < 0 || rank >= p->nparts) return bad("bad partition or rank");
  const auto &R = p->ranks[rank];
  auto put = [](int32_t *dst, const std::vector<int32_t> &v) {
    if (dst && !v.empty()) std::memcpy(dst, v.data(), v.size() * sizeof(int32_t));
  };
  put(ia, R.ia);
  put(ja, R.ja);
  put(src, R.jsrc);
  if (l2g) {
    put(l2g, R.rows);
    if (!R.ghosts.empty())
      std::memcpy(l2g + R.rows.size(), R.ghosts.data(), R.ghosts.size() * sizeof(int32_t));
  }
  put(iaSends, R.ia_snd);
  put(iaRcvs, R.ia_rcv);
  put(fMap, R.fmap);
  if (vizPart)
    for (size_t n = 0; n < R.viz.size(); ++n) vizPart[n] = static_cast<int16_t>(R.viz[n]);
  return SFR_OK;
}

int sfr_part_destroy(sfr_part *p) {
  delete p;
  return SFR_OK;
}

}  // extern "C"
