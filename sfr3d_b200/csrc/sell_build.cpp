// Host conversion of the reference's sparse layouts into the device SELL-32
// layout.  Each row keeps the reference's summation order:
//   CSRD unsym  (matVecCsrD, HccaBlas.c:3358-3400): entries in stored order;
//   CSRD/CSRC sym and CSRC unsym (matVecCsrDSym HccaBlas.c:2620-2655,
//     matVecCsrC HccaBlas.c:4223-4258): the row's own strict-lower entries in
//     stored order, then the mirrored entries y[j] += a*x[i] of later rows i
//     in increasing i -- the order the reference's scatter adds them;
//   ELLPACK (matVecEllPack, HccaBlas.c:4700-4755): the row's slots in order,
//     padded slots included.
// The diagonal is kept apart and summed first, as every reference kernel
// does.  The transpose, when asked for, orders each row diagonal first and
// then by increasing column.
#include <algorithm>
#include <climits>
#include <cstdint>
#include <string>
#include <vector>

#include "internal.h"

namespace sfr {

namespace {

struct RowLists {
  std::vector<int64_t> ptr;  // n + 1
  std::vector<int32_t> col;
  std::vector<int32_t> src;
};

int fail(std::string *why, const std::string &msg) {
  if (why) *why = msg;
  return SFR_BAD_INPUT;
}

// false when the slot count does not fit int32 offsets
bool to_sell(int32_t n, const RowLists &rl, HostSell *h) {
  h->n = n;
  h->nslices = (n + kWarpHost - 1) / kWarpHost;
  h->sptr.assign(h->nslices + 1, 0);
  int32_t maxw = 0;
  int64_t total = 0;
  for (int32_t s = 0; s < h->nslices; ++s) {
    int64_t w = 0;
    for (int32_t l = 0; l < kWarpHost; ++l) {
      const int32_t r = s * kWarpHost + l;
      if (r < n) w = std::max<int64_t>(w, rl.ptr[r + 1] - rl.ptr[r]);
    }
    maxw = std::max<int32_t>(maxw, static_cast<int32_t>(w));
    total += w * kWarpHost;
    if (total > INT32_MAX) return false;
    h->sptr[s + 1] = static_cast<int32_t>(total);
  }
  h->max_width = maxw;
  const int64_t nslots = h->sptr[h->nslices];
  h->col.assign(nslots, 0);
  h->src.assign(nslots, -1);
  int32_t band = 0;
  int64_t nnz = 0;
  for (int32_t s = 0; s < h->nslices; ++s) {
    const int32_t base = h->sptr[s];
    const int32_t w = (h->sptr[s + 1] - base) / kWarpHost;
    for (int32_t l = 0; l < kWarpHost; ++l) {
      const int32_t r = s * kWarpHost + l;
      const int64_t len = r < n ? rl.ptr[r + 1] - rl.ptr[r] : 0;
      for (int32_t k = 0; k < w; ++k) {
        const int64_t e = base + static_cast<int64_t>(k) * kWarpHost + l;
        if (k < len) {
          const int32_t c = rl.col[rl.ptr[r] + k];
          h->col[e] = c;
          h->src[e] = rl.src[rl.ptr[r] + k];
          band = std::max(band, c > r ? c - r : r - c);
          ++nnz;
        } else {
          h->col[e] = r < n ? r : 0;
          h->src[e] = -1;
        }
      }
    }
  }
  h->bandwidth = band;
  h->nnz = nnz;
  return true;
}

}  // namespace

int build_sell(int32_t neq, int32_t nad, const int32_t *ia, const int32_t *ja,
               int32_t storage, int32_t unsym, HostSell *a, HostSell *at,
               int32_t *nsrc, std::string *why) {
  (void)nad;
  if (neq <= 0) return fail(why, "neq must be positive");
  if (!ia) return fail(why, "ia is NULL");
  RowLists rl;
  rl.ptr.assign(static_cast<size_t>(neq) + 1, 0);

  if (storage == SFR_ELLPACK) {
    const int32_t width = ia[0];
    if (width < 0 || width > 1024) return fail(why, "ELLPACK width out of range");
    if (static_cast<int64_t>(ia[1]) != static_cast<int64_t>(neq) * width)
      return fail(why, "ELLPACK header ia[1] != neq*width");
    const int64_t total = static_cast<int64_t>(neq) * width;
    if (total > INT32_MAX) return fail(why, "too many ELLPACK slots");
    if (width > 0 && !ja) return fail(why, "ja is NULL");
    rl.col.resize(total);
    rl.src.resize(total);
    for (int32_t i = 0; i < neq; ++i) {
      rl.ptr[i + 1] = rl.ptr[i] + width;
      for (int32_t k = 0; k < width; ++k) {
        const int64_t q = static_cast<int64_t>(i) * width + k;
        const int32_t c = ja[q];
        if (c < 0 || c >= neq) return fail(why, "ja out of range");
        rl.col[q] = c;
        rl.src[q] = static_cast<int32_t>(q);
      }
    }
    *nsrc = static_cast<int32_t>(total);
  } else if (storage == SFR_CSRD || storage == SFR_CSRC) {
    const int32_t base = ia[0];
    if (base < 0) return fail(why, "ia[0] negative");
    for (int32_t i = 0; i < neq; ++i)
      if (ia[i + 1] < ia[i]) return fail(why, "ia not monotone");
    const int64_t cnt = static_cast<int64_t>(ia[neq]) - base;
    if (cnt > 0 && !ja) return fail(why, "ja is NULL");
    for (int64_t k = 0; k < cnt; ++k)
      if (ja[base + k] < 0 || ja[base + k] >= neq) return fail(why, "ja out of range");
    const bool full = storage == SFR_CSRD && unsym;
    if (full) {
      rl.col.resize(cnt);
      rl.src.resize(cnt);
      for (int32_t i = 0; i < neq; ++i) {
        rl.ptr[i + 1] = ia[i + 1] - base;
        for (int32_t k = ia[i]; k < ia[i + 1]; ++k) {
          rl.col[k - base] = ja[k];
          rl.src[k - base] = k - base;
        }
      }
      *nsrc = static_cast<int32_t>(cnt);
    } else {
      // strict-lower storage; the upper half is the mirror (sym) or au
      for (int32_t i = 0; i < neq; ++i)
        for (int32_t k = ia[i]; k < ia[i + 1]; ++k)
          if (ja[k] >= i) return fail(why, "entry not strictly lower in lower-triangular storage");
      const bool use_au = storage == SFR_CSRC && unsym;
      if (use_au && 2 * cnt > INT32_MAX) return fail(why, "too many entries");
      std::vector<int64_t> up_cnt(static_cast<size_t>(neq) + 1, 0);
      for (int64_t k = 0; k < cnt; ++k) ++up_cnt[ja[base + k] + 1];
      for (int32_t j = 0; j < neq; ++j) up_cnt[j + 1] += up_cnt[j];
      std::vector<int32_t> up_col(cnt), up_src(cnt);
      std::vector<int64_t> fillp(up_cnt.begin(), up_cnt.end() - 1);
      for (int32_t i = 0; i < neq; ++i)
        for (int32_t k = ia[i]; k < ia[i + 1]; ++k) {
          const int32_t j = ja[k];
          const int64_t q = fillp[j]++;
          up_col[q] = i;
          up_src[q] = static_cast<int32_t>((k - base) + (use_au ? cnt : 0));
        }
      rl.col.resize(2 * cnt);
      rl.src.resize(2 * cnt);
      int64_t q = 0;
      for (int32_t i = 0; i < neq; ++i) {
        for (int32_t k = ia[i]; k < ia[i + 1]; ++k) {
          rl.col[q] = ja[k];
          rl.src[q] = k - base;
          ++q;
        }
        for (int64_t u = up_cnt[i]; u < up_cnt[i + 1]; ++u) {
          rl.col[q] = up_col[u];
          rl.src[q] = up_src[u];
          ++q;
        }
        rl.ptr[i + 1] = q;
      }
      *nsrc = static_cast<int32_t>(use_au ? 2 * cnt : cnt);
    }
  } else {
    return fail(why, "storage must be CSRD (2), CSRC (3) or ELLPACK (4)");
  }
  if (!to_sell(neq, rl, a)) return fail(why, "system too large for int32 slot offsets");

  if (at) {
    // transpose: entries (i, c, src) -> row c, ordered by increasing i
    RowLists tl;
    tl.ptr.assign(static_cast<size_t>(neq) + 1, 0);
    for (size_t q = 0; q < rl.col.size(); ++q) ++tl.ptr[rl.col[q] + 1];
    for (int32_t j = 0; j < neq; ++j) tl.ptr[j + 1] += tl.ptr[j];
    tl.col.resize(rl.col.size());
    tl.src.resize(rl.col.size());
    std::vector<int64_t> fillp(tl.ptr.begin(), tl.ptr.end() - 1);
    for (int32_t i = 0; i < neq; ++i)
      for (int64_t q = rl.ptr[i]; q < rl.ptr[i + 1]; ++q) {
        const int32_t c = rl.col[q];
        const int64_t t = fillp[c]++;
        tl.col[t] = i;
        tl.src[t] = rl.src[q];
      }
    if (!to_sell(neq, tl, at)) return fail(why, "system too large for int32 slot offsets");
  }
  return SFR_OK;
}

}  // namespace sfr
