/* CPU restatement of the split tree's treelet restructuring. TEST INFRASTRUCTURE ONLY.
 *
 * The checker for cuda-path-tracer_b200/csrc/split.cu k_treelet (CPT_SPLIT_TREELET), an
 * extension without a reference counterpart: the optimisation of Karras and Aila, "Fast
 * Parallel Construction of High-Quality Bounding Volume Hierarchies" (HPG 2013), which the
 * reference's README cites and does not implement. tests/ compare the product's
 * restructured records with this restatement byte for byte; the product never links,
 * loads or calls this file.
 *
 * Input: the split tree's 96-B records (two 40-B child slots, the Node word
 * (left << 2 | right internal << 1 | left internal), the right child's index, two more
 * words), n leaves and the leaves' boxes by leaf index. One round: nodes are visited
 * children first; a node with at least gamma leaves gets its treelet — its two children,
 * then, up to 7 leaves, the internal treelet leaf of largest half surface area (the first
 * such leaf on ties) replaced by its two children — and the topology over the treelet's
 * leaves that minimises the summed half area of its internal nodes, found over all
 * subsets with ties to the smallest (cost bits, split mask); it replaces the old one when
 * cheaper by more than a factor 0.999999 and no taller, in the treelet's own nodes (the
 * first created node is the root, the next ones in the order the top-down rebuild
 * creates them, left child before right). Rewritten records get 0 in their last two
 * words. All arithmetic is float, one rounding per operation (-ffp-contract=off).
 */
#include <float.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define TL_LEAVES 7
#define TL_SUBSETS (1 << TL_LEAVES)

typedef struct {
    float* rec;
    const float* leaf_boxes;
    uint32_t n, gamma;
    uint32_t* size;
    uint32_t* height;
    int bad;
} tl_tree;

static inline uint32_t f2u(float f) { uint32_t u; memcpy(&u, &f, 4); return u; }
static inline float u2f(uint32_t u) { float f; memcpy(&f, &u, 4); return f; }

static inline float half_area(const float* b)
{
    float dx = b[3] - b[0], dy = b[4] - b[1], dz = b[5] - b[2];
    float s = dx * dy + dy * dz;
    return s + dz * dx;
}

static inline uint32_t popc(uint32_t x) { return (uint32_t)__builtin_popcount(x); }

typedef struct {
    float box[TL_LEAVES][6];
    float slot[TL_LEAVES][10];
    uint32_t id[TL_LEAVES], size[TL_LEAVES], height[TL_LEAVES];
    uint32_t inode[TL_LEAVES - 1];
    uint32_t internal_mask, m;
    float old_cost;
} tl_form;

/* treelet leaves k0, k1 := the children of internal node q */
static int take_children(tl_tree* t, uint32_t q, int k0, int k1, tl_form* f)
{
    const float* r = t->rec + 24 * (size_t)q;
    uint32_t word = f2u(r[20]);
    uint32_t ids[2] = {word >> 2, f2u(r[21])};
    for (int side = 0; side < 2; ++side) {
        int k = side ? k1 : k0;
        int internal = (word >> side) & 1u;
        uint32_t id = ids[side];
        if (internal ? id >= t->n - 1 : id >= t->n) return 0;
        memcpy(f->slot[k], r + 10 * side, 10 * sizeof(float));
        if (internal) {
            memcpy(f->box[k], r + 10 * side, 6 * sizeof(float));
            f->size[k] = t->size[id];
            f->height[k] = t->height[id];
            f->internal_mask |= 1u << k;
        } else {
            memcpy(f->box[k], t->leaf_boxes + 6 * (size_t)id, 6 * sizeof(float));
            f->size[k] = 1;
            f->height[k] = 0;
            f->internal_mask &= ~(1u << k);
        }
        f->id[k] = id;
    }
    return 1;
}

static void treelet(tl_tree* t, uint32_t r, uint32_t h_before)
{
    tl_form f;
    memset(&f, 0, sizeof(f));
    f.inode[0] = r;
    if (!take_children(t, r, 0, 1, &f)) { t->bad = 1; return; }
    uint32_t m = 2, ni = 1;
    float rb[6];
    for (int a = 0; a < 3; ++a) {
        rb[a] = f.box[0][a] < f.box[1][a] ? f.box[0][a] : f.box[1][a];
        rb[3 + a] = f.box[0][3 + a] > f.box[1][3 + a] ? f.box[0][3 + a] : f.box[1][3 + a];
    }
    float old = half_area(rb);
    while (m < TL_LEAVES) {
        int b = -1;
        float ba = -1.f;
        for (uint32_t k = 0; k < m; ++k)
            if ((f.internal_mask >> k) & 1u) {
                float a = half_area(f.box[k]);
                if (a > ba) { ba = a; b = (int)k; }
            }
        if (b < 0) break;
        uint32_t q = f.id[b];
        f.inode[ni++] = q;
        old = old + ba;
        if (!take_children(t, q, b, (int)m, &f)) { t->bad = 1; return; }
        ++m;
    }
    if (m < 3) return;
    const uint32_t full = (1u << m) - 1u;
    float c[TL_SUBSETS];
    uint8_t split[TL_SUBSETS];
    for (uint32_t S = 1; S <= full; ++S) {
        if (popc(S) == 1) { c[S] = 0.f; continue; }
        float b[6] = {FLT_MAX, FLT_MAX, FLT_MAX, -FLT_MAX, -FLT_MAX, -FLT_MAX};
        for (uint32_t k = 0; k < m; ++k)
            if ((S >> k) & 1u)
                for (int a = 0; a < 3; ++a) {
                    if (f.box[k][a] < b[a]) b[a] = f.box[k][a];
                    if (f.box[k][3 + a] > b[3 + a]) b[3 + a] = f.box[k][3 + a];
                }
        c[S] = half_area(b);
    }
    for (uint32_t k = 2; k <= m; ++k)
        for (uint32_t S = 1; S <= full; ++S) {
            if (popc(S) != k) continue;
            uint32_t low = S & (0u - S);
            uint64_t best = ~0ull;
            for (uint32_t P = (S - 1) & S; P; P = (P - 1) & S) {
                if (!(P & low)) continue;
                float v = c[P] + c[S ^ P];
                uint64_t key = ((uint64_t)f2u(v) << 32) | P;
                if (key < best) best = key;
            }
            c[S] = c[S] + u2f((uint32_t)(best >> 32));
            split[S] = (uint8_t)(best & 127u);
        }
    float limit = old * 0.999999f;
    if (!(c[full] < limit)) return;
    uint32_t sub[TL_LEAVES - 1], ck[TL_LEAVES - 1][2], cnt = 1;
    sub[0] = full;
    for (uint32_t j = 0; j < cnt; ++j) {
        uint32_t S = sub[j], P = split[S];
        uint32_t X[2] = {P, S ^ P};
        for (int side = 0; side < 2; ++side) {
            if (X[side] == 0u || (X[side] & ~S)) { t->bad = 1; return; }
            if (popc(X[side]) == 1) {
                ck[j][side] = (uint32_t)__builtin_ctz(X[side]);
            } else {
                if (cnt >= m - 1) { t->bad = 1; return; }
                sub[cnt] = X[side];
                ck[j][side] = 8u + cnt;
                ++cnt;
            }
        }
    }
    if (cnt != m - 1) { t->bad = 1; return; }
    uint32_t h[TL_LEAVES - 1], sz[TL_LEAVES - 1];
    for (int j = (int)cnt - 1; j >= 0; --j) {
        uint32_t hh = 0, ss = 0;
        for (int side = 0; side < 2; ++side) {
            uint32_t cc = ck[j][side];
            uint32_t hc = cc < 8u ? f.height[cc] : h[cc - 8u];
            hh = hc > hh ? hc : hh;
            ss += cc < 8u ? f.size[cc] : sz[cc - 8u];
        }
        h[j] = hh + 1u;
        sz[j] = ss;
    }
    if (h[0] > h_before) return;
    for (uint32_t j = 0; j < cnt; ++j) {
        uint32_t nd = f.inode[j];
        float* rec = t->rec + 24 * (size_t)nd;
        uint32_t ids[2], word = 0;
        for (int side = 0; side < 2; ++side) {
            uint32_t cc = ck[j][side];
            float slot[10];
            if (cc < 8u) {
                ids[side] = f.id[cc];
                memcpy(slot, f.slot[cc], sizeof(slot));
                if ((f.internal_mask >> cc) & 1u) word |= 1u << side;
            } else {
                uint32_t x = cc - 8u, X = sub[x];
                ids[side] = f.inode[x];
                word |= 1u << side;
                for (int a = 0; a < 3; ++a) { slot[a] = FLT_MAX; slot[3 + a] = -FLT_MAX; }
                for (uint32_t k = 0; k < m; ++k)
                    if ((X >> k) & 1u)
                        for (int a = 0; a < 3; ++a) {
                            if (f.box[k][a] < slot[a]) slot[a] = f.box[k][a];
                            if (f.box[k][3 + a] > slot[3 + a]) slot[3 + a] = f.box[k][3 + a];
                        }
                slot[6] = slot[7] = slot[8] = slot[9] = 0.0f;
            }
            memcpy(rec + 10 * side, slot, sizeof(slot));
        }
        word |= ids[0] << 2;
        rec[20] = u2f(word);
        rec[21] = u2f(ids[1]);
        rec[22] = 0.0f;
        rec[23] = 0.0f;
        t->size[nd] = sz[j];
        t->height[nd] = h[j];
    }
}

/* children first: sizes and heights from the (final) children, then the node's treelet */
static void visit(tl_tree* t, uint32_t node, int depth)
{
    if (t->bad || depth > 4096) { t->bad = 1; return; }
    const float* r = t->rec + 24 * (size_t)node;
    uint32_t word = f2u(r[20]);
    uint32_t ids[2] = {word >> 2, f2u(r[21])};
    uint32_t size = 0, height = 0;
    for (int side = 0; side < 2; ++side) {
        if ((word >> side) & 1u) {
            if (ids[side] >= t->n - 1) { t->bad = 1; return; }
            visit(t, ids[side], depth + 1);
            if (t->bad) return;
            size += t->size[ids[side]];
            if (t->height[ids[side]] > height) height = t->height[ids[side]];
        } else {
            if (ids[side] >= t->n) { t->bad = 1; return; }
            size += 1;
        }
    }
    t->size[node] = size;
    t->height[node] = height + 1;
    if (size >= t->gamma) treelet(t, node, height + 1);
}

/* One round of treelet restructuring of the records (n - 1 of them, rewritten in place).
 * leaf_boxes: n x 6 floats (lo xyz, hi xyz) by leaf index. Returns 0, or -1 for a
 * malformed tree (an index out of range, a cycle deeper than 4096). */
int orc_treelet(float* records, uint32_t n, const float* leaf_boxes, uint32_t gamma)
{
    if (n < 2 || !records || !leaf_boxes) return -1;
    tl_tree t;
    t.rec = records;
    t.leaf_boxes = leaf_boxes;
    t.n = n;
    t.gamma = gamma;
    t.size = (uint32_t*)calloc(n, sizeof(uint32_t));
    t.height = (uint32_t*)calloc(n, sizeof(uint32_t));
    t.bad = 0;
    if (!t.size || !t.height) { free(t.size); free(t.height); return -1; }
    if (n >= 3) visit(&t, 0, 0);
    free(t.size);
    free(t.height);
    return t.bad ? -1 : 0;
}
