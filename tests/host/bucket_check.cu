// Host-side check of the bucket ranking of gpz_b200/csrc/gpz_encode.cuh
// (rank_buckets): its schedule emulated lane by lane on the CPU -- shared
// atomics in an arbitrary arrival order, the bucket scan, placement at bucket
// start + slot, a full sort of every bucket of kEncSmall or more points (the
// warp's bitonic network), then the odd-even transposition steps between
// neighbouring positions of one bucket, with the pair across lanes -- and
// compared with a plain sort of the composites (block id - kmin) << 10 | r.
// The transposition runs ceil(largest bucket / 2) rounds, at most 8; an
// exhaustive check confirms that n alternating steps sort n values whichever
// parity comes first.  Also checks that a chunk is declined exactly when it
// has a big bucket.  Compiled with nvcc, runs on the CPU.
#include <algorithm>
#include <cstdio>
#include <cstdint>
#include <vector>
#include "gpz_encode.cuh"

static uint64_t s = 0x2545F4914F6CDD1Dull;
static uint32_t rnd() { s ^= s << 13; s ^= s >> 7; s ^= s << 17; return (uint32_t)s; }

struct Out {
  bool declined = false;
  int steps = 0;  // transposition rounds that ran
  uint32_t id[1024], r[1024];
};

// ids[l][j]: block id of lane l's register j (point 32j + l, rank r = 32l + j).
// narrow: composites of at most 32 bits (1024 buckets, whole composites in S,
// steps compare values alone, a chunk with a big bucket is declined);
// otherwise the wide form (2048 buckets, the bits below the bucket in S, the
// bucket of each position beside).
static Out emulate(const uint32_t (&ids)[32][32], uint32_t nvalid, bool narrow) {
  Out o;
  const bool full = nvalid == 1024u;
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0;
  for (int l = 0; l < 32; ++l)
    for (int j = 0; j < 32; ++j)
      if (32u * j + l < nvalid) { kmin = std::min(kmin, ids[l][j]); kmax = std::max(kmax, ids[l][j]); }
  const unsigned long long cmax = ((unsigned long long)(kmax - kmin) << 10) | 1023ull;
  uint32_t cbits = 0;
  while ((cmax >> cbits) != 0) ++cbits;
  cbits = std::max(cbits, 21u);
  const uint32_t shb = cbits - gpzb::kEncBucketBits, lowb = shb - 10u;
  uint32_t vv[32][32], b[32][32], slot[32][32];
  std::vector<uint32_t> cnt(2048, 0);
  // counting: program order over j, lanes of one j in a random order
  for (int j = 0; j < 32; ++j) {
    int perm[32];
    for (int l = 0; l < 32; ++l) perm[l] = l;
    for (int l = 31; l > 0; --l) std::swap(perm[l], perm[rnd() % (l + 1)]);
    for (int t = 0; t < 32; ++t) {
      const int l = perm[t];
      const uint32_t koff = ids[l][j] - kmin;
      if (narrow) {  // 1024 buckets on the top 10 bits
        vv[l][j] = (koff << 10) | (32u * l + j);
        b[l][j] = vv[l][j] >> (shb + 1u);
      } else {
        b[l][j] = koff >> lowb;
        vv[l][j] = ((koff & ((1u << lowb) - 1u)) << 10) | (32u * l + j);
      }
      if (full || 32u * j + l < nvalid) slot[l][j] = cnt[b[l][j]]++;
    }
  }
  bool big = false;
  for (uint32_t k = 0; k < 2048; ++k) big |= cnt[k] >= (uint32_t)gpzb::kEncSmall;
  if (narrow && big) { o.declined = true; return o; }
  std::vector<uint32_t> start(2049, 0);
  for (uint32_t k = 0; k < 2048; ++k) start[k + 1] = start[k] + cnt[k];
  uint32_t S[1024], B[1024];
  for (int i = 0; i < 1024; ++i) { S[i] = rnd(); B[i] = rnd() % 2048; }  // stale words
  for (int l = 0; l < 32; ++l)
    for (int j = 0; j < 32; ++j)
      if (full || 32u * j + l < nvalid) {
        const uint32_t pos = start[b[l][j]] + slot[l][j];
        S[pos] = vv[l][j];
        B[pos] = b[l][j];
      }
  for (uint32_t k = 0; k < 2048; ++k)
    if (cnt[k] >= (uint32_t)gpzb::kEncSmall) std::sort(S + start[k], S + start[k + 1]);
  uint32_t key[32][32], bpos[32][32];
  for (int l = 0; l < 32; ++l)
    for (int j = 0; j < 32; ++j) {
      const bool valid = full || 32u * l + j < nvalid;
      key[l][j] = narrow && !valid ? 0xFFFFFFFFu : S[32 * l + j];
      bpos[l][j] = narrow ? 0u : valid ? B[32 * l + j] : (0x80000000u | (32u * l + j));
    }
  // rounds: ceil(largest bucket / 2), at most 8 (bigger buckets are sorted)
  uint32_t maxb = 0;
  for (uint32_t k = 0; k < 2048; ++k) maxb = std::max(maxb, cnt[k]);
  const uint32_t rounds = std::min((maxb + 1u) >> 1, (uint32_t)gpzb::kEncSmall / 2u);
  for (uint32_t it = 0; it < rounds; ++it) {
    ++o.steps;
    for (int l = 0; l < 32; ++l)
      for (int j = 0; j < 32; j += 2)
        if (bpos[l][j] == bpos[l][j + 1] && key[l][j] > key[l][j + 1]) std::swap(key[l][j], key[l][j + 1]);
    uint32_t nk[32], nb[32], pk[32], pb[32];
    for (int l = 0; l < 32; ++l) {  // the shuffles read before the odd step
      nk[l] = key[(l + 1) & 31][0]; nb[l] = bpos[(l + 1) & 31][0];
      pk[l] = key[(l + 31) & 31][31]; pb[l] = bpos[(l + 31) & 31][31];
    }
    for (int l = 0; l < 32; ++l)
      for (int j = 1; j < 31; j += 2)
        if (bpos[l][j] == bpos[l][j + 1] && key[l][j] > key[l][j + 1]) std::swap(key[l][j], key[l][j + 1]);
    bool xr[32], xl[32];
    for (int l = 0; l < 32; ++l) {
      xr[l] = l < 31 && nb[l] == bpos[l][31] && key[l][31] > nk[l];
      xl[l] = l > 0 && pb[l] == bpos[l][0] && pk[l] > key[l][0];
    }
    for (int l = 0; l < 32; ++l) {
      if (xr[l]) key[l][31] = nk[l];
      if (xl[l]) key[l][0] = pk[l];
    }
  }
  for (int l = 0; l < 32; ++l)
    for (int j = 0; j < 32; ++j) {
      o.id[32 * l + j] = narrow ? kmin + (key[l][j] >> 10) : kmin + ((bpos[l][j] << lowb) | (key[l][j] >> 10));
      o.r[32 * l + j] = key[l][j] & 1023u;
    }
  return o;
}

// Emulates one chunk and compares it with a plain sort; returns the mismatches.
static long check(const uint32_t (&ids)[32][32], uint32_t nvalid, long &declined, long &maxsteps) {
  uint32_t kmin = 0xFFFFFFFFu, kmax = 0;
  for (int l = 0; l < 32; ++l)
    for (int j = 0; j < 32; ++j)
      if (32u * j + l < nvalid) { kmin = std::min(kmin, ids[l][j]); kmax = std::max(kmax, ids[l][j]); }
  const bool wide = ((unsigned long long)(kmax - kmin) << 10 | 1023ull) >> 32 != 0;
  const Out o = emulate(ids, nvalid, !wide);
  if (o.declined) {  // the warp sort ranks it (checked in network_check)
    ++declined;
    return 0;
  }
  long bad = 0;
  maxsteps = std::max<long>(maxsteps, o.steps);
  std::vector<unsigned long long> ref;
  for (int l = 0; l < 32; ++l)
    for (int j = 0; j < 32; ++j)
      if (32u * j + l < nvalid) ref.push_back(((unsigned long long)(ids[l][j] - kmin) << 10) | (32u * l + j));
  std::sort(ref.begin(), ref.end());
  for (uint32_t p = 0; p < nvalid; ++p)
    bad += o.id[p] != kmin + (uint32_t)(ref[p] >> 10) || o.r[p] != (uint32_t)(ref[p] & 1023u);
  return bad;
}

// n alternating odd / even transposition steps sort n values, whichever parity
// comes first: every permutation of n <= 9 distinct values.
static long exhaustive_steps() {
  long bad = 0;
  for (int n = 1; n <= 9; ++n) {
    int p[9];
    for (int i = 0; i < n; ++i) p[i] = i;
    do {
      for (int first = 0; first < 2; ++first) {
        int a[9];
        std::copy(p, p + n, a);
        for (int step = 0; step < n; ++step)
          for (int i = (first + step) & 1; i + 1 < n; i += 2)
            if (a[i] > a[i + 1]) std::swap(a[i], a[i + 1]);
        for (int i = 0; i < n; ++i) bad += a[i] != i;
      }
    } while (std::next_permutation(p, p + n));
  }
  return bad;
}

int main() {
  long bad = exhaustive_steps(), checks = 0, declined = 0, maxsteps = 0;
  for (int it = 0; it < 20000; ++it) {
    uint32_t ids[32][32];
    const int kind = it % 5;
    const uint32_t nvalid = it % 7 == 0 ? 1 + rnd() % 1024 : 1024;
    const uint32_t base = rnd() & 0x3FFFFFFFu;
    for (int l = 0; l < 32; ++l)
      for (int j = 0; j < 32; ++j) {
        uint32_t v;
        if (kind == 0) v = rnd() & 0x7FFFFFFFu;                       // ids over 2^31: wide composites
        else if (kind == 1) v = base + rnd() % (1u << 22);             // 32-bit composites
        else if (kind == 2) v = base + (rnd() % 4 == 0 ? rnd() % 40 : rnd() % (1u << 21));  // one dense region
        else if (kind == 3) v = base + rnd() % 3000;                   // narrow range, many duplicates
        else v = (rnd() % 8 == 0) ? (rnd() & 0x7FFFFFFFu) : base + rnd() % 64;  // wide with big buckets
        ids[l][j] = v & 0x7FFFFFFFu;
      }
    bad += check(ids, nvalid, declined, maxsteps);
    ++checks;
  }
  // the longest small bucket, 15 points with descending ids across a lane
  // boundary, in many arrival orders
  for (int it = 0; it < 2000; ++it) {
    uint32_t ids[32][32];
    for (int l = 0; l < 32; ++l)
      for (int j = 0; j < 32; ++j) ids[l][j] = (uint32_t)(32 * l + j) * 4096u;  // one point per bucket
    for (int t = 0; t < 15; ++t) {  // ranks 25..39 share one bucket, ids descending;
      const int rr = 25 + t;         // 26 smaller ids put them at positions 26..40
      ids[rr / 32][rr % 32] = 40u * 4096u + 3000u - (uint32_t)t;
    }
    bad += check(ids, 1024, declined, maxsteps);
    ++checks;
  }
  printf("checks=%ld declined=%ld max_steps=%ld bad=%ld\n", checks, declined, maxsteps, bad);
  return bad != 0 || declined == 0 || maxsteps > gpzb::kEncSmall / 2;
}
