/*
 * gsoracle.c - CPU ORACLE for the gpusketch_b200 test suite.  TEST INFRASTRUCTURE ONLY.
 *
 * This is a plain-C restatement of the reference's sketch arithmetic and Boruvka emulation,
 * used by tests/ (and by bench.py's cpu_baseline leg) as the checker.  The product never
 * links, loads or calls anything in this directory.
 *
 * Each function cites the reference file:line it follows (paths inside the reference
 * project).  The 8-byte XXH3 path restates the published xxHash algorithm
 * (XXH3_len_4to8_64b + rrmxmx, xxHash >= 0.8.0, whose 64-bit output is frozen); the
 * reference links the external `xxhash` target (CMakeLists.txt:123) without pinning a
 * version.  Pinned by tests/golden/xxh3_vectors.json (made with python-xxhash 3.7.0 /
 * libxxhash 0.8.2) and by the reference's own sources compiled into oracle/_ref.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <math.h>

#define OR_GOOD 0
#define OR_ZERO 1
#define OR_FAIL 2

/* ---------------- hash (include/types.h:8-9, include/bucket.h:54-63) ---------------- */

static uint64_t or_rotl64(uint64_t x, int r) { return (x << r) | (x >> (64 - r)); }

/* XXH3_64bits_withSeed(&key, 8, seed) for a little-endian u64 key. */
uint64_t or_xxh3_8(uint64_t key, uint64_t seed) {
  const uint64_t secret_8_24 = 0x1cad21f72c81017cULL ^ 0xdb979083e96dd4deULL; /* kSecret[8..24) */
  const uint64_t mx2 = 0x9FB21C651E98DF25ULL;
  uint32_t lo = (uint32_t)seed;
  uint32_t sw = ((lo & 0xffu) << 24) | ((lo & 0xff00u) << 8) | ((lo >> 8) & 0xff00u) | (lo >> 24);
  uint64_t s = seed ^ ((uint64_t)sw << 32);
  uint64_t bitflip = secret_8_24 - s;
  uint64_t input64 = (key >> 32) + ((key & 0xffffffffULL) << 32);
  uint64_t h = input64 ^ bitflip;
  h ^= or_rotl64(h, 49) ^ or_rotl64(h, 24);
  h *= mx2;
  h ^= (h >> 35) + 8;
  h *= mx2;
  return h ^ (h >> 28);
}

/* Bucket_Boruvka::get_index_depth (include/bucket.h:54-59). */
uint32_t or_index_depth(uint64_t e, uint64_t seed_and_col, uint32_t max_depth) {
  uint64_t h = or_xxh3_8(e, seed_and_col) | (1ULL << max_depth);
  return (uint32_t)__builtin_ctzll(h);
}

/* concat_pairing_fn (src/util.cpp:45-51). */
uint64_t or_concat(uint32_t i, uint32_t j) {
  if (i > j) { uint32_t t = i; i = j; j = t; }
  return ((uint64_t)i << 32) | j;
}

/* ---------------- sizing (include/sketch.h:177-191,312-320; src/sketch.cpp:24-30) ---------------- */

/* out: [num_samples, cols_per_sample, num_columns, bkt_per_col, num_buckets] */
void or_geometry(uint32_t V, double factor, uint32_t out[5]) {
  double vec_len = ceil((double)V * (V - 1) / 2);                 /* calc_vector_length */
  /* calc_vector_length returns vec_t (u64); the sizing then runs on the integer value */
  uint64_t vlen = (uint64_t)vec_len;
  size_t samples = (size_t)ceil(factor * log2((double)V) / (1 - 0.263034406));
  if (samples < 18) samples = 18;                                  /* calc_cc_samples */
  size_t bkt = (size_t)(ceil(log2((double)vlen)) + 1);             /* calc_bkt_per_col */
  if (bkt % 16 == 0) bkt += 1;
  out[0] = (uint32_t)samples;
  out[1] = 1;                                                      /* default_cols_per_sample */
  out[2] = (uint32_t)samples;
  out[3] = (uint32_t)bkt;
  out[4] = (uint32_t)(samples * bkt + 1);
}

/* ---------------- sketch update / sample / merge (src/sketch.cpp) ---------------- */

/* Sketch::update, CameoSketch branch (src/sketch.cpp:85-99).  sk = 2*nb u64 (alpha,gamma). */
void or_sketch_update(uint64_t* sk, uint32_t num_columns, uint32_t bkt, uint32_t nb,
                      uint64_t seed, uint64_t e) {
  uint64_t cs = or_xxh3_8(e, seed);
  sk[2 * (nb - 1)] ^= e;
  sk[2 * (nb - 1) + 1] ^= cs;
  for (uint32_t c = 0; c < num_columns; c++) {
    uint32_t d = or_index_depth(e, seed + 5ULL * c, bkt);
    if (d < bkt) {
      size_t id = (size_t)c * bkt + d;
      sk[2 * id] ^= e;
      sk[2 * id + 1] ^= cs;
    }
  }
}

/* CCSketchAlg::update for each record: both endpoint sketches (src/cc_sketch_alg.cpp:154-160). */
void or_ingest_pairs(uint64_t* sketches, uint32_t V, uint32_t num_columns, uint32_t bkt, uint32_t nb,
                     uint64_t seed, const uint32_t* pairs, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) {
    uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
    if (a >= V || b >= V) continue;
    uint64_t e = or_concat(a, b);
    or_sketch_update(sketches + (size_t)a * nb * 2, num_columns, bkt, nb, seed, e);
    or_sketch_update(sketches + (size_t)b * nb * 2, num_columns, bkt, nb, seed, e);
  }
}

/* Min-cut ingest: each record goes to subgraph levels 0..min(tag, num_levels-1) with
 * tag = get_index_depth(e, seed, L-1) (src/mc_gpu_sketch_alg.cpp:157-169,83-137). */
void or_ingest_pairs_levels(uint64_t* sketches, uint32_t V, uint32_t num_levels, uint32_t L,
                            uint32_t num_columns, uint32_t bkt, uint32_t nb, uint64_t seed,
                            const uint32_t* pairs, uint64_t n) {
  for (uint64_t i = 0; i < n; i++) {
    uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
    if (a >= V || b >= V) continue;
    uint64_t e = or_concat(a, b);
    uint32_t tag = or_index_depth(e, seed, L - 1);
    uint32_t top = tag < num_levels - 1 ? tag : num_levels - 1;
    for (uint32_t g = 0; g <= top; g++) {
      uint64_t* base = sketches + (size_t)g * V * nb * 2;
      or_sketch_update(base + (size_t)a * nb * 2, num_columns, bkt, nb, seed, e);
      or_sketch_update(base + (size_t)b * nb * 2, num_columns, bkt, nb, seed, e);
    }
  }
}

static int or_is_good(uint64_t alpha, uint64_t gamma, uint64_t seed) {
  return gamma == or_xxh3_8(alpha, seed);                           /* include/bucket.h:65-67 */
}

/* Sketch::sample for one column (cols_per_sample = 1) (src/sketch.cpp:110-132).
 * col_buckets points at the column's bkt buckets, det at the deterministic bucket. */
int or_sample(const uint64_t* col_buckets, const uint64_t* det, uint32_t bkt, uint64_t seed,
              uint64_t* idx) {
  if (det[0] == 0 && det[1] == 0) { *idx = 0; return OR_ZERO; }
  if (or_is_good(det[0], det[1], seed)) { *idx = det[0]; return OR_GOOD; }
  for (uint32_t j = 0; j < bkt; j++) {
    if (or_is_good(col_buckets[2 * j], col_buckets[2 * j + 1], seed)) {
      *idx = col_buckets[2 * j]; return OR_GOOD;
    }
  }
  *idx = 0;
  return OR_FAIL;
}

/* ---------------- DSU (include/dsu.h); partitions only, roots are free ---------------- */

static uint32_t or_find(uint32_t* p, uint32_t x) {
  while (p[x] != x) { p[x] = p[p[x]]; x = p[x]; }
  return x;
}
static int or_union(uint32_t* p, uint32_t a, uint32_t b) {
  a = or_find(p, a); b = or_find(p, b);
  if (a == b) return 0;
  if (a < b) p[b] = a; else p[a] = b;     /* smaller id becomes the root */
  return 1;
}

/*
 * Boruvka emulation (CCSketchAlg::boruvka_emulation / perform_boruvka_round / run_round_zero /
 * sample_supernode / create_merge_instructions, src/cc_sketch_alg.cpp:164-540).
 *
 * Round 0 samples every vertex sketch at column `round0_col` (0 for connected components;
 * MCSketchAlg's run_k_round_zero samples the stored sketches whose sample_idx advances once
 * per forest, so forest j of a subgraph uses column j, src/mc_sketch_alg.cpp:307-328).
 * Round r > 0 XORs column r and the deterministic bucket of every member of each current
 * component (Sketch::range_merge, src/sketch.cpp:172-195) and samples column r.  The sampled
 * edges of a round are unioned after the round; the partition does not depend on that order.
 * A round r >= num_samples throws OutOfSamplesException in the reference (range_merge puts the
 * sketch in a fail state, src/sketch.cpp:173-177,111-113): returns -1 then.
 * Forest edges (src<dst) are the sampled edges whose union merged two components, taken in
 * ascending component-root order.
 */
int or_boruvka(const uint64_t* sketches, uint32_t V, uint32_t num_samples, uint32_t bkt,
               uint32_t nb, uint64_t seed, uint32_t round0_col, uint32_t* labels,
               uint32_t* rounds_out, uint32_t* forest, uint64_t* n_forest) {
  uint32_t* parent = (uint32_t*)malloc(sizeof(uint32_t) * V);
  uint32_t* root_of = (uint32_t*)malloc(sizeof(uint32_t) * V);
  uint64_t* acc = (uint64_t*)malloc(sizeof(uint64_t) * 2 * (size_t)(bkt + 1) * V);
  uint64_t* samp = (uint64_t*)malloc(sizeof(uint64_t) * V);
  int* res = (int*)malloc(sizeof(int) * V);
  uint64_t nf = 0;
  int status = 0;
  for (uint32_t i = 0; i < V; i++) parent[i] = i;
  uint32_t round = 0;
  for (;;) {
    int modified = 0;
    if (round == 0) {
      if (round0_col >= num_samples) { status = -1; break; }
      for (uint32_t v = 0; v < V; v++) {
        const uint64_t* sk = sketches + (size_t)v * nb * 2;
        res[v] = or_sample(sk + (size_t)round0_col * bkt * 2, sk + (size_t)(nb - 1) * 2, bkt, seed,
                           &samp[v]);
      }
      for (uint32_t v = 0; v < V; v++) root_of[v] = v;
    } else {
      if (round >= num_samples) { status = -1; break; }
      for (uint32_t v = 0; v < V; v++) root_of[v] = or_find(parent, v);
      memset(acc, 0, sizeof(uint64_t) * 2 * (size_t)(bkt + 1) * V);
      for (uint32_t v = 0; v < V; v++) {
        const uint64_t* sk = sketches + (size_t)v * nb * 2;
        uint64_t* a = acc + (size_t)root_of[v] * (bkt + 1) * 2;
        const uint64_t* col = sk + (size_t)round * bkt * 2;
        for (uint32_t j = 0; j < 2 * bkt; j++) a[j] ^= col[j];
        a[2 * bkt] ^= sk[(size_t)(nb - 1) * 2];
        a[2 * bkt + 1] ^= sk[(size_t)(nb - 1) * 2 + 1];
      }
      for (uint32_t v = 0; v < V; v++) {
        if (root_of[v] != v) { res[v] = -1; continue; }
        const uint64_t* a = acc + (size_t)v * (bkt + 1) * 2;
        res[v] = or_sample(a, a + 2 * bkt, bkt, seed, &samp[v]);
      }
    }
    for (uint32_t v = 0; v < V; v++) {
      if (res[v] == OR_FAIL) modified = 1;
      else if (res[v] == OR_GOOD) {
        uint32_t s = (uint32_t)(samp[v] >> 32), d = (uint32_t)samp[v];
        if (s >= V || d >= V) continue;   /* a checksum collision would yield a bogus edge */
        if (or_union(parent, s, d)) {
          modified = 1;
          if (forest) { forest[2 * nf] = s; forest[2 * nf + 1] = d; }
          nf++;
        }
      }
    }
    if (!modified) break;
    round++;
  }
  for (uint32_t v = 0; v < V; v++) labels[v] = or_find(parent, v);
  if (rounds_out) *rounds_out = round;
  if (n_forest) *n_forest = nf;
  free(parent); free(root_of); free(acc); free(samp); free(res);
  return status;
}

/*
 * k edge-disjoint spanning forests of one subgraph (MCSketchAlg::calc_disjoint_spanning_forests
 * and filter_sf_edges, src/mc_sketch_alg.cpp:837-919): forest j runs Boruvka with round-0 column
 * first_col + j, then XORs its edges out of both endpoint sketches; at the end every forest is
 * XORed back in.  `sketches` is modified in place and restored.  forests: k * 2*(V-1) u32.
 * Returns -1 if a forest ran out of samples (the reference throws), else 0.
 */
int or_k_forests(uint64_t* sketches, uint32_t V, uint32_t num_samples, uint32_t num_columns,
                 uint32_t bkt, uint32_t nb, uint64_t seed, uint32_t k, uint32_t first_col,
                 uint32_t* forests, uint64_t* sizes) {
  uint32_t* labels = (uint32_t*)malloc(sizeof(uint32_t) * V);
  int status = 0;
  uint32_t done = 0;
  for (uint32_t j = 0; j < k; j++) {
    uint32_t* f = forests + (size_t)j * 2 * (V > 0 ? V - 1 : 0);
    uint32_t rounds;
    if (or_boruvka(sketches, V, num_samples, bkt, nb, seed, first_col + j, labels, &rounds, f,
                   &sizes[j]) != 0) { status = -1; sizes[j] = 0; break; }
    for (uint64_t i = 0; i < sizes[j]; i++) {
      uint64_t e = or_concat(f[2 * i], f[2 * i + 1]);
      or_sketch_update(sketches + (size_t)f[2 * i] * nb * 2, num_columns, bkt, nb, seed, e);
      or_sketch_update(sketches + (size_t)f[2 * i + 1] * nb * 2, num_columns, bkt, nb, seed, e);
    }
    done++;
  }
  for (uint32_t j = 0; j < done; j++) {
    uint32_t* f = forests + (size_t)j * 2 * (V > 0 ? V - 1 : 0);
    for (uint64_t i = 0; i < sizes[j]; i++) {
      uint64_t e = or_concat(f[2 * i], f[2 * i + 1]);
      or_sketch_update(sketches + (size_t)f[2 * i] * nb * 2, num_columns, bkt, nb, seed, e);
      or_sketch_update(sketches + (size_t)f[2 * i + 1] * nb * 2, num_columns, bkt, nb, seed, e);
    }
  }
  free(labels);
  return status;
}

/* ---------------- exact models (test/util/graph_verifier.cpp:49-80) ---------------- */

static int or_cmp_u64(const void* a, const void* b) {
  uint64_t x = *(const uint64_t*)a, y = *(const uint64_t*)b;
  return x < y ? -1 : (x > y);
}

/* Final edge set of a toggle stream (each record flips {src,dst}; self-loops ignored).
 * Writes the surviving edges as (src<dst) pairs into out (capacity n pairs); returns count. */
uint64_t or_final_edges(uint32_t V, const uint32_t* pairs, uint64_t n, uint32_t* out) {
  uint64_t* ids = (uint64_t*)malloc(sizeof(uint64_t) * (n ? n : 1));
  uint64_t m = 0;
  for (uint64_t i = 0; i < n; i++) {
    uint32_t a = pairs[2 * i], b = pairs[2 * i + 1];
    if (a == b || a >= V || b >= V) continue;
    ids[m++] = or_concat(a, b);
  }
  qsort(ids, m, sizeof(uint64_t), or_cmp_u64);
  uint64_t k = 0;
  for (uint64_t i = 0; i < m;) {
    uint64_t j = i;
    while (j < m && ids[j] == ids[i]) j++;
    if ((j - i) & 1) { out[2 * k] = (uint32_t)(ids[i] >> 32); out[2 * k + 1] = (uint32_t)ids[i]; k++; }
    i = j;
  }
  free(ids);
  return k;
}

/* Exact connected components of an edge list (Kruskal DSU of GraphVerifier::kruskal).
 * labels[v] = minimum vertex id of v's component; returns the component count. */
uint32_t or_cc_of_edges(uint32_t V, const uint32_t* edges, uint64_t m, uint32_t* labels) {
  uint32_t* p = (uint32_t*)malloc(sizeof(uint32_t) * V);
  for (uint32_t i = 0; i < V; i++) p[i] = i;
  uint32_t ncc = V;
  for (uint64_t i = 0; i < m; i++) ncc -= (uint32_t)or_union(p, edges[2 * i], edges[2 * i + 1]);
  for (uint32_t v = 0; v < V; v++) labels[v] = or_find(p, v);
  free(p);
  return ncc;
}

/* Exact global minimum cut (Stoer-Wagner, dense O(V^3)); the reference calls VieCut
 * (src/mc_sketch_alg.cpp:966-1002), which is not in the reference tree.  For test sizes only.
 * side[v] = 1 on one side of the returned cut.  Returns UINT64_MAX for V < 2. */
uint64_t or_stoer_wagner(uint32_t V, const uint32_t* edges, uint64_t m, uint8_t* side) {
  if (V < 2) return UINT64_MAX;
  uint64_t* w = (uint64_t*)calloc((size_t)V * V, sizeof(uint64_t));
  for (uint64_t i = 0; i < m; i++) {
    uint32_t a = edges[2 * i], b = edges[2 * i + 1];
    if (a == b) continue;
    w[(size_t)a * V + b]++; w[(size_t)b * V + a]++;
  }
  uint32_t* vert = (uint32_t*)malloc(sizeof(uint32_t) * V);   /* active super vertices */
  uint32_t* grp = (uint32_t*)malloc(sizeof(uint32_t) * V);    /* vertex -> super vertex */
  uint64_t* key = (uint64_t*)malloc(sizeof(uint64_t) * V);
  uint8_t* added = (uint8_t*)malloc(V);
  for (uint32_t i = 0; i < V; i++) { vert[i] = i; grp[i] = i; }
  uint32_t n = V;
  uint64_t best = UINT64_MAX;
  uint32_t best_t = 0;
  uint32_t* best_members = (uint32_t*)malloc(sizeof(uint32_t) * V);
  uint8_t* cur_side = (uint8_t*)malloc(V);
  while (n > 1) {
    memset(added, 0, V);
    for (uint32_t i = 0; i < n; i++) key[vert[i]] = 0;
    uint32_t prev = vert[0], last = vert[0];
    added[vert[0]] = 1;
    for (uint32_t i = 0; i < n; i++) key[vert[i]] = w[(size_t)vert[0] * V + vert[i]];
    for (uint32_t it = 1; it < n; it++) {
      uint32_t sel = UINT32_MAX; uint64_t bk = 0;
      for (uint32_t i = 0; i < n; i++) {
        uint32_t x = vert[i];
        if (!added[x] && (sel == UINT32_MAX || key[x] > bk)) { sel = x; bk = key[x]; }
      }
      added[sel] = 1;
      prev = last; last = sel;
      if (it == n - 1) {
        if (bk < best) {
          best = bk; best_t = sel;
          for (uint32_t v = 0; v < V; v++) cur_side[v] = (grp[v] == sel);
          memcpy(best_members, grp, sizeof(uint32_t) * V);
        }
      }
      for (uint32_t i = 0; i < n; i++) {
        uint32_t x = vert[i];
        if (!added[x]) key[x] += w[(size_t)sel * V + x];
      }
    }
    /* merge last into prev */
    for (uint32_t i = 0; i < n; i++) {
      uint32_t x = vert[i];
      w[(size_t)prev * V + x] += w[(size_t)last * V + x];
      w[(size_t)x * V + prev] = w[(size_t)prev * V + x];
    }
    w[(size_t)prev * V + prev] = 0;
    for (uint32_t v = 0; v < V; v++) if (grp[v] == last) grp[v] = prev;
    for (uint32_t i = 0; i < n; i++) if (vert[i] == last) { vert[i] = vert[n - 1]; break; }
    n--;
  }
  (void)best_t;
  if (side) memcpy(side, cur_side, V);
  free(w); free(vert); free(grp); free(key); free(added); free(best_members); free(cur_side);
  return best;
}
