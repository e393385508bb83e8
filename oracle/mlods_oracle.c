/*
 * mlods_oracle.c -- TEST INFRASTRUCTURE ONLY.
 *
 * A double-precision CPU restatement of the reference's point-set surface
 * projection path (CorentinMercier/MlodSurfaces, sources/apss and
 * sources/dual-contouring).  It is the checker the parity tests, the smoke
 * test and the benchmark's CPU baseline compare against; the product path
 * (mlodsurfaces_b200, libmlods.so) never links, loads or calls it.
 *
 * What it restates, function by function (paths inside the reference project):
 *   - octree build: recursive midpoint split (float sum of the float bounds, halved in double), child
 *     boxes stored as float, 1 point per leaf, depth <= max_depth, child slot
 *     c = xi + 2 yi + 4 zi                     sources/apss/CPUUtils.cpp:271-329
 *   - tight root box                            sources/apss/CPUUtils.cpp:571-579
 *   - per-sample areas diag(leaf)^2/#pts        sources/apss/CPUUtils.cpp:236-252
 *   - bottom-up moment sums                     sources/apss/CPUUtils.cpp:358-398
 *   - breadth-first numbering                   sources/apss/CPUUtils.cpp:601-619
 *   - father/firstChild/nextBrother links       sources/apss/CPUUtils.cpp:213-234
 *   - weight kernels                            sources/apss/Kernel.cpp:64-83 (CPU),
 *                                               sources/apss/GPUUtils.cu:243-257 (GPU)
 *   - MLoD traversal, GPU blend rule            sources/apss/Fastapss.cu:160-333
 *   - MLoD traversal, CPU blend rule            sources/apss/CPUUtils.cpp:443-513
 *   - blend s = (1 - cos(3.14159265 t)) / 2     sources/apss/Fastapss.cu:84-95,
 *                                               sources/apss/CPUUtils.cpp:400-408
 *   - algebraic sphere fit + projection         sources/apss/Fastapss.cu:335-396 (GPU),
 *                                               sources/apss/CPUUtils.cpp:739-782 (CPU)
 *   - global (all points) APSS                  sources/apss/CPUUtils.cpp:515-528,
 *                                               sources/apss/GlobalAPSS.cu:113-168
 *   - kNN / ball APSS                           sources/apss/CPUUtils.cpp:690-737,
 *                                               sources/dual-contouring/kdTreeNN/kdTreeNN.h:416-490
 *   - DC corner field f = (c - proj).n          sources/scene/scene.cpp:1361-1394
 *   - DC vertex with the zero normal field      sources/dual-contouring/dual_contouring.h:91-176
 *
 * Differences from the reference, all deliberate:
 *   - Every sum, weight and solve runs in double; moments are kept centred on
 *     the node centroid so that far-from-origin clouds do not cancel.
 *   - A point lying exactly on a split goes to the low child (the reference
 *     draws rand(), CPUUtils.cpp:299-308); ties are counted and reported.
 *   - Multi-point leaves (depth == max_depth) are summed in the GPU rule, as
 *     Fastapss.cu:191-200 intends (the reference kernel indexes its per-depth
 *     array out of bounds there); the CPU rule keeps the reference's
 *     last-point-only overwrite (CPUUtils.cpp:453-456).
 *
 * Build: gcc -O2 -ffp-contract=off -fPIC -shared -fopenmp (oracle/Makefile).
 */
#include <float.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_PI_REF 3.14159265 /* the reference's literal, Fastapss.cu:93 */

enum { ORC_GAUSSIAN = 0, ORC_SINGULAR = 1, ORC_GAUSSIAN_MULTIPLE = 2 }; /* Kernel.h:37 */
enum { ORC_RULE_GPU = 0, ORC_RULE_CPU = 1 };

typedef struct {
    int type;
    double sigma, exponent, shift;
    int nsig;
    const double* sigmas; /* the caller's array, any length (Kernel::sigmas is a std::vector) */
} orc_kernel;

/* ---------------------------------------------------------------- tree */

typedef struct {
    int64_t n_pts;
    int max_depth;
    float* pts; /* 3 n */
    float* nrm; /* 3 n */
    double* area; /* n */
    int64_t n_nodes;
    /* per node, breadth-first order */
    int32_t* depth;
    int32_t* parent;
    int32_t* first_child;
    int32_t* n_children;
    int32_t* next_brother;
    int32_t* leaf_off; /* offset into perm, -1 for internal nodes */
    int32_t* leaf_cnt; /* 0 for internal nodes */
    int32_t* slot; /* child slot inside the parent, -1 for the root */
    float* bmin; /* 3 per node */
    float* bmax;
    /* centred moments in double: M0, pbar[3], Mn[3], Cpn, Cpp */
    double* mom; /* 9 per node */
    int32_t* perm; /* leaf point lists, leaves in breadth-first order */
    int64_t n_ties;
} orc_tree;

typedef struct {
    float bb[3], BB[3];
    int depth;
    int32_t child[8];
    int32_t seg_s, seg_e; /* point segment in the work index array (leaves) */
} bnode;

typedef struct {
    bnode* v;
    int64_t n, cap;
} bnode_vec;

static int32_t bnode_new(bnode_vec* nv)
{
    if (nv->n == nv->cap) {
        nv->cap = nv->cap ? nv->cap * 2 : 1024;
        nv->v = (bnode*)realloc(nv->v, (size_t)nv->cap * sizeof(bnode));
    }
    bnode* b = &nv->v[nv->n];
    memset(b, 0, sizeof(*b));
    for (int c = 0; c < 8; ++c) b->child[c] = -1;
    b->seg_s = b->seg_e = -1;
    return (int32_t)nv->n++;
}

/* Recursive midpoint split, CPUUtils.cpp:271-329.  idx[s,e) are the node's
 * points in ascending original order; the partition is stable. */
static void build_rec(bnode_vec* nv, int32_t id, const float* pts, int32_t* idx, int32_t* tmp,
                      int32_t s, int32_t e, int depth, int max_depth, int64_t* ties)
{
    nv->v[id].depth = depth;
    if (e - s <= 1 || depth == max_depth) {
        nv->v[id].seg_s = s;
        nv->v[id].seg_e = e;
        return;
    }
    float bb[3], BB[3];
    memcpy(bb, nv->v[id].bb, sizeof bb);
    memcpy(BB, nv->v[id].BB, sizeof BB);
    double split[3];
    /* the reference's `(bb[0] + BB[0]) / 2.0` (CPUUtils.cpp:286-288): the two
     * float bounds are added in float, then halved in double */
    for (int a = 0; a < 3; ++a) split[a] = (double)(float)(bb[a] + BB[a]) / 2.0;
    int32_t cnt[8] = {0};
    unsigned char* slot = (unsigned char*)malloc((size_t)(e - s));
    for (int32_t i = s; i < e; ++i) {
        const float* p = pts + 3 * (int64_t)idx[i];
        int c = 0;
        for (int a = 0; a < 3; ++a) {
            double pa = (double)p[a];
            if (pa == split[a]) ++*ties; /* tie: stays low (see header) */
            if (pa > split[a]) c |= 1 << a;
        }
        slot[i - s] = (unsigned char)c;
        cnt[c]++;
    }
    int32_t off[9];
    off[0] = s;
    for (int c = 0; c < 8; ++c) off[c + 1] = off[c] + cnt[c];
    int32_t pos[8];
    for (int c = 0; c < 8; ++c) pos[c] = off[c];
    for (int32_t i = s; i < e; ++i) tmp[pos[slot[i - s]]++] = idx[i];
    memcpy(idx + s, tmp + s, (size_t)(e - s) * sizeof(int32_t));
    free(slot);
    /* children are created for xi outer, yi, zi inner (CPUUtils.cpp:314-327);
     * creation order does not change slots or breadth-first numbering. */
    for (int xi = 0; xi < 2; ++xi)
        for (int yi = 0; yi < 2; ++yi)
            for (int zi = 0; zi < 2; ++zi) {
                int c = xi + 2 * yi + 4 * zi;
                if (cnt[c] == 0) continue;
                int32_t ch = bnode_new(nv);
                int sel[3] = {xi, yi, zi};
                for (int a = 0; a < 3; ++a) {
                    double lo = sel[a] ? split[a] : (double)bb[a];
                    double hi = sel[a] ? (double)BB[a] : split[a];
                    nv->v[ch].bb[a] = (float)lo;
                    nv->v[ch].BB[a] = (float)hi;
                }
                nv->v[id].child[c] = ch;
                build_rec(nv, ch, pts, idx, tmp, off[c], off[c + 1], depth + 1, max_depth, ties);
            }
}

static void merge_moments(const double* a, const double* b, double* out)
{
    /* parallel-axis merge of two centred moment sets */
    double M = a[0] + b[0];
    double pb[3];
    for (int k = 0; k < 3; ++k) pb[k] = (a[0] * a[1 + k] + b[0] * b[1 + k]) / M;
    double cpn = a[7] + b[7], cpp = a[8] + b[8];
    for (int s = 0; s < 2; ++s) {
        const double* m = s ? b : a;
        double d[3] = {m[1] - pb[0], m[2] - pb[1], m[3] - pb[2]};
        cpn += d[0] * m[4] + d[1] * m[5] + d[2] * m[6];
        cpp += m[0] * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
    }
    out[0] = M;
    for (int k = 0; k < 3; ++k) out[1 + k] = pb[k];
    for (int k = 0; k < 3; ++k) out[4 + k] = a[4 + k] + b[4 + k];
    out[7] = cpn;
    out[8] = cpp;
}

orc_tree* orc_tree_build(const float* pts, const float* nrm, int64_t n, int max_depth)
{
    if (n <= 0 || max_depth < 0 || max_depth > 20) return NULL;
    orc_tree* t = (orc_tree*)calloc(1, sizeof(orc_tree));
    t->n_pts = n;
    t->max_depth = max_depth;
    t->pts = (float*)malloc((size_t)n * 3 * sizeof(float));
    t->nrm = (float*)malloc((size_t)n * 3 * sizeof(float));
    memcpy(t->pts, pts, (size_t)n * 3 * sizeof(float));
    memcpy(t->nrm, nrm, (size_t)n * 3 * sizeof(float));

    bnode_vec nv = {0};
    int32_t root = bnode_new(&nv);
    for (int a = 0; a < 3; ++a) nv.v[root].bb[a] = nv.v[root].BB[a] = pts[a];
    for (int64_t i = 1; i < n; ++i)
        for (int a = 0; a < 3; ++a) {
            float v = pts[3 * i + a];
            if (v < nv.v[root].bb[a]) nv.v[root].bb[a] = v;
            if (v > nv.v[root].BB[a]) nv.v[root].BB[a] = v;
        }
    int32_t* idx = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    int32_t* tmp = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    for (int64_t i = 0; i < n; ++i) idx[i] = (int32_t)i;
    build_rec(&nv, root, pts, idx, tmp, 0, (int32_t)n, 0, max_depth, &t->n_ties);
    free(tmp);

    /* breadth-first numbering, children visited in slot order (CPUUtils.cpp:601-619) */
    int64_t nn = nv.n;
    t->n_nodes = nn;
    int32_t* order = (int32_t*)malloc((size_t)nn * sizeof(int32_t)); /* bfs -> build id */
    int32_t* bfs_of = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    int64_t head = 0, tail = 0;
    order[tail++] = root;
    while (head < tail) {
        int32_t id = order[head++];
        for (int c = 0; c < 8; ++c)
            if (nv.v[id].child[c] >= 0) order[tail++] = nv.v[id].child[c];
    }
    for (int64_t b = 0; b < nn; ++b) bfs_of[order[b]] = (int32_t)b;

    t->depth = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->parent = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->first_child = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->n_children = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->next_brother = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->leaf_off = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->leaf_cnt = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->slot = (int32_t*)malloc((size_t)nn * sizeof(int32_t));
    t->bmin = (float*)malloc((size_t)nn * 3 * sizeof(float));
    t->bmax = (float*)malloc((size_t)nn * 3 * sizeof(float));
    t->mom = (double*)calloc((size_t)nn * 9, sizeof(double));
    t->perm = (int32_t*)malloc((size_t)n * sizeof(int32_t));
    t->area = (double*)malloc((size_t)n * sizeof(double));
    for (int64_t b = 0; b < nn; ++b) {
        t->parent[b] = -1;
        t->next_brother[b] = -1;
        t->slot[b] = -1;
    }
    int32_t perm_pos = 0;
    for (int64_t b = 0; b < nn; ++b) {
        const bnode* nd = &nv.v[order[b]];
        t->depth[b] = nd->depth;
        memcpy(t->bmin + 3 * b, nd->bb, 3 * sizeof(float));
        memcpy(t->bmax + 3 * b, nd->BB, 3 * sizeof(float));
        int32_t first = -1, prev = -1, nc = 0;
        for (int c = 0; c < 8; ++c) {
            if (nd->child[c] < 0) continue;
            int32_t cb = bfs_of[nd->child[c]];
            t->parent[cb] = (int32_t)b;
            t->slot[cb] = c;
            if (first < 0) first = cb;
            if (prev >= 0) t->next_brother[prev] = cb;
            prev = cb;
            ++nc;
        }
        t->first_child[b] = first;
        t->n_children[b] = nc;
        if (nc == 0) {
            int32_t cnt = nd->seg_e - nd->seg_s;
            t->leaf_off[b] = perm_pos;
            t->leaf_cnt[b] = cnt;
            memcpy(t->perm + perm_pos, idx + nd->seg_s, (size_t)cnt * sizeof(int32_t));
            perm_pos += cnt;
        } else {
            t->leaf_off[b] = -1;
            t->leaf_cnt[b] = 0;
        }
    }
    free(order);
    free(bfs_of);
    free(idx);
    free(nv.v);

    /* per-sample area (CPUUtils.cpp:236-252) and leaf moments */
    for (int64_t b = 0; b < nn; ++b) {
        if (t->leaf_cnt[b] == 0) continue;
        double d2 = 0.0;
        for (int a = 0; a < 3; ++a) {
            double e = (double)t->bmax[3 * b + a] - (double)t->bmin[3 * b + a];
            d2 += e * e;
        }
        int32_t cnt = t->leaf_cnt[b];
        double ar = d2 / cnt;
        double* m = t->mom + 9 * b;
        double sp[3] = {0, 0, 0}, sa = 0;
        for (int32_t k = 0; k < cnt; ++k) {
            int32_t i = t->perm[t->leaf_off[b] + k];
            t->area[i] = ar;
            sa += ar;
            for (int a = 0; a < 3; ++a) sp[a] += ar * (double)t->pts[3 * i + a];
        }
        m[0] = sa;
        for (int a = 0; a < 3; ++a) m[1 + a] = sp[a] / sa;
        for (int32_t k = 0; k < cnt; ++k) {
            int32_t i = t->perm[t->leaf_off[b] + k];
            double d[3], nn3[3];
            for (int a = 0; a < 3; ++a) {
                d[a] = (double)t->pts[3 * i + a] - m[1 + a];
                nn3[a] = (double)t->nrm[3 * i + a];
                m[4 + a] += ar * nn3[a];
            }
            m[7] += ar * (d[0] * nn3[0] + d[1] * nn3[1] + d[2] * nn3[2]);
            m[8] += ar * (d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
        }
    }
    /* internal nodes: deepest first (breadth-first order reversed) */
    for (int64_t b = nn - 1; b >= 0; --b) {
        if (t->n_children[b] == 0) continue;
        double acc[9];
        int32_t c0 = t->first_child[b];
        memcpy(acc, t->mom + 9 * (int64_t)c0, sizeof acc);
        for (int32_t c = c0 + 1; c < c0 + t->n_children[b]; ++c) merge_moments(acc, t->mom + 9 * (int64_t)c, acc);
        memcpy(t->mom + 9 * b, acc, sizeof acc);
    }
    return t;
}

void orc_tree_free(orc_tree* t)
{
    if (!t) return;
    free(t->pts); free(t->nrm); free(t->area);
    free(t->depth); free(t->parent); free(t->first_child); free(t->n_children);
    free(t->next_brother); free(t->leaf_off); free(t->leaf_cnt); free(t->slot);
    free(t->bmin); free(t->bmax); free(t->mom); free(t->perm);
    free(t);
}

int64_t orc_tree_num_nodes(const orc_tree* t) { return t->n_nodes; }
int64_t orc_tree_num_ties(const orc_tree* t) { return t->n_ties; }

void orc_tree_export(const orc_tree* t, int32_t* depth, int32_t* parent, int32_t* first_child,
                     int32_t* n_children, int32_t* next_brother, int32_t* leaf_off, int32_t* leaf_cnt,
                     int32_t* perm, float* bmin, float* bmax, double* mom, double* area)
{
    int64_t nn = t->n_nodes;
    if (depth) memcpy(depth, t->depth, (size_t)nn * 4);
    if (parent) memcpy(parent, t->parent, (size_t)nn * 4);
    if (first_child) memcpy(first_child, t->first_child, (size_t)nn * 4);
    if (n_children) memcpy(n_children, t->n_children, (size_t)nn * 4);
    if (next_brother) memcpy(next_brother, t->next_brother, (size_t)nn * 4);
    if (leaf_off) memcpy(leaf_off, t->leaf_off, (size_t)nn * 4);
    if (leaf_cnt) memcpy(leaf_cnt, t->leaf_cnt, (size_t)nn * 4);
    if (perm) memcpy(perm, t->perm, (size_t)t->n_pts * 4);
    if (bmin) memcpy(bmin, t->bmin, (size_t)nn * 12);
    if (bmax) memcpy(bmax, t->bmax, (size_t)nn * 12);
    if (mom) memcpy(mom, t->mom, (size_t)nn * 9 * sizeof(double));
    if (area) memcpy(area, t->area, (size_t)t->n_pts * sizeof(double));
}

/* ---------------------------------------------------------------- kernels */

static void kernel_from_args(orc_kernel* k, int type, double sigma, double exponent, double shift,
                             const double* sigmas, int nsig)
{
    k->type = type;
    k->sigma = sigma;
    k->exponent = exponent;
    k->shift = shift;
    k->nsig = nsig;
    k->sigmas = sigmas;
}

/* Kernel::w (Kernel.cpp:64-83) and KernelGPU::w (GPUUtils.cu:243-257), in double. */
static double kernel_w(const orc_kernel* k, double d2, int rule)
{
    if (k->type == ORC_GAUSSIAN_MULTIPLE) {
        double s = 0.0;
        for (int i = 0; i < k->nsig; ++i) {
            double sg = k->sigmas[i];
            s += exp(-d2 / (2.0 * sg * sg)) / (sg * sg * sg);
        }
        if (rule == ORC_RULE_CPU && s == 0.0) s = k->shift;
        return s;
    }
    if (k->type == ORC_GAUSSIAN) return exp(-d2 / (2.0 * k->sigma * k->sigma)) + k->shift;
    if (k->type == ORC_SINGULAR) {
        double v = k->shift > 1e-4 ? k->shift : 1e-4;
        return pow(v, k->exponent) / pow(d2 + k->shift, k->exponent);
    }
    return 1.0;
}

/* ---------------------------------------------------------------- projection */

typedef struct {
    const orc_tree* t;
    const orc_kernel* k;
    int rule;
    double cutoff;
    int min_depth;
    double q[3];
    int64_t visited;
} mlod_ctx;

static inline double dist3(const double* a, const double* b)
{
    double x = a[0] - b[0], y = a[1] - b[1], z = a[2] - b[2];
    return sqrt(x * x + y * y + z * z);
}

static void node_center_radius(const orc_tree* t, int64_t b, double c[3], double* r)
{
    double d2 = 0.0;
    for (int a = 0; a < 3; ++a) {
        double lo = t->bmin[3 * b + a], hi = t->bmax[3 * b + a];
        c[a] = (lo + hi) / 2.0;
        d2 += (hi - lo) * (hi - lo);
    }
    *r = sqrt(d2) / 2.0;
}

/* acc[9] in the query frame: Sw, Sn[3], Sp[3] (p-q), Spn, Spp. */
static void add_moments(double* acc, const double* m, const double* q, double coef)
{
    double d[3] = {m[1] - q[0], m[2] - q[1], m[3] - q[2]};
    double d2 = d[0] * d[0] + d[1] * d[1] + d[2] * d[2];
    acc[0] += coef * m[0];
    for (int a = 0; a < 3; ++a) acc[1 + a] += coef * m[4 + a];
    for (int a = 0; a < 3; ++a) acc[4 + a] += coef * m[0] * d[a];
    acc[7] += coef * (m[7] + d[0] * m[4] + d[1] * m[5] + d[2] * m[6]);
    acc[8] += coef * (m[8] + d2 * m[0]);
}

static void add_point(double* acc, const orc_tree* t, int32_t i, const double* q, double coef)
{
    double m[9];
    m[0] = t->area[i];
    for (int a = 0; a < 3; ++a) {
        m[1 + a] = t->pts[3 * i + a];
        m[4 + a] = t->area[i] * (double)t->nrm[3 * i + a];
    }
    m[7] = 0.0;
    m[8] = 0.0;
    add_moments(acc, m, q, coef);
}

static double wdist2(const double* p, const double* q)
{
    double x = p[0] - q[0], y = p[1] - q[1], z = p[2] - q[2];
    return x * x + y * y + z * z;
}

static void mlod_rec(mlod_ctx* cx, int64_t b, double* acc)
{
    const orc_tree* t = cx->t;
    cx->visited++;
    if (t->leaf_cnt[b] > 0) {
        int32_t cnt = t->leaf_cnt[b];
        int32_t k0 = (cx->rule == ORC_RULE_CPU) ? cnt - 1 : 0; /* CPUUtils.cpp:453-456 overwrite */
        for (int32_t k = k0; k < cnt; ++k) {
            int32_t i = t->perm[t->leaf_off[b] + k];
            double p[3] = {t->pts[3 * i], t->pts[3 * i + 1], t->pts[3 * i + 2]};
            double w = kernel_w(cx->k, wdist2(p, cx->q), cx->rule);
            add_point(acc, t, i, cx->q, w);
        }
        return;
    }
    const double* m = t->mom + 9 * b;
    if (t->depth[b] >= cx->min_depth) {
        double c[3], r;
        node_center_radius(t, b, c, &r);
        double dist = dist3(cx->q, c);
        double w = kernel_w(cx->k, wdist2(m + 1, cx->q), cx->rule);
        if (dist > cx->cutoff * r) {
            add_moments(acc, m, cx->q, w);
            return;
        }
        double dP = fabs(dist - r * cx->cutoff);
        int32_t c0 = t->first_child[b], nc = t->n_children[b];
        for (int32_t ch = c0; ch < c0 + nc; ++ch) {
            double cc[3], rc;
            node_center_radius(t, ch, cc, &rc);
            double dC = dist3(cx->q, cc) - rc * cx->cutoff;
            if (dC < 0.0) dC = 0.0;
            double tt = dP / (dP + dC);
            double beta = (1.0 - cos(ORC_PI_REF * tt)) / 2.0;
            double child[9] = {0};
            mlod_rec(cx, ch, child);
            for (int a = 0; a < 9; ++a) acc[a] += beta * child[a];
            double wp = (cx->rule == ORC_RULE_GPU) ? w * t->mom[9 * (int64_t)ch] / m[0] : w / (double)nc;
            add_moments(acc, m, cx->q, (1.0 - beta) * wp);
        }
        return;
    }
    int32_t c0 = t->first_child[b], nc = t->n_children[b];
    for (int32_t ch = c0; ch < c0 + nc; ++ch) mlod_rec(cx, ch, acc);
}

static void normalize3(double* v, int zero_safe)
{
    double n = sqrt(v[0] * v[0] + v[1] * v[1] + v[2] * v[2]);
    if (n != 0.0 || !zero_safe) {
        v[0] /= n; v[1] /= n; v[2] /= n;
    } else {
        v[0] = v[1] = v[2] = 0.0;
    }
}

/* Sphere fit + projection of the frame origin (the query) from query-frame
 * sums.  Fastapss.cu:354-395 (GPU: |u4|<1e-6, zero-safe normalize) and
 * CPUUtils.cpp:744-781 (CPU: |u4|<1e-12, glm::normalize).  Returns 1 when the
 * result was NaN (output = query, normal = 0). */
static int fit_and_project(const double* acc, double u4_thr, int zero_safe, double step_max, double* x,
                           double* nrm)
{
    double Sw = acc[0];
    const double* Sn = acc + 1;
    const double* Sp = acc + 4;
    double Spn = acc[7], Spp = acc[8];
    double u4 = 0.5 * (Spn - (Sp[0] * Sn[0] + Sp[1] * Sn[1] + Sp[2] * Sn[2]) / Sw) /
                (Spp - (Sp[0] * Sp[0] + Sp[1] * Sp[1] + Sp[2] * Sp[2]) / Sw);
    double u123[3];
    for (int a = 0; a < 3; ++a) u123[a] = (Sn[a] - 2.0 * u4 * Sp[a]) / Sw;
    double u0 = -((Sp[0] * u123[0] + Sp[1] * u123[1] + Sp[2] * u123[2]) + u4 * Spp) / Sw;
    x[0] = x[1] = x[2] = 0.0;
    if (fabs(u4) < u4_thr) {
        double nv[3] = {-u123[0], -u123[1], -u123[2]};
        double l2 = nv[0] * nv[0] + nv[1] * nv[1] + nv[2] * nv[2];
        double lambda = u0 / l2;
        for (int a = 0; a < 3; ++a) x[a] = lambda * nv[a];
        for (int a = 0; a < 3; ++a) nrm[a] = Sn[a];
        normalize3(nrm, zero_safe);
    } else {
        double c[3];
        for (int a = 0; a < 3; ++a) c[a] = u123[a] / (-2.0 * u4);
        double r2 = c[0] * c[0] + c[1] * c[1] + c[2] * c[2] - u0 / u4;
        double rad = sqrt(r2 > 0.0 ? r2 : 0.0);
        double pc[3] = {-c[0], -c[1], -c[2]};
        normalize3(pc, zero_safe);
        for (int a = 0; a < 3; ++a) x[a] = c[a] + rad * pc[a];
        for (int a = 0; a < 3; ++a) nrm[a] = u123[a] + 2.0 * u4 * x[a];
        normalize3(nrm, zero_safe);
    }
    if (isnan(x[0]) || isnan(x[1]) || isnan(x[2])) {
        x[0] = x[1] = x[2] = 0.0;
        nrm[0] = nrm[1] = nrm[2] = 0.0;
        return 1;
    }
    double step = sqrt(x[0] * x[0] + x[1] * x[1] + x[2] * x[2]);
    if (step > step_max)
        for (int a = 0; a < 3; ++a) x[a] *= step_max / step;
    return 0;
}

double orc_tree_radius(const orc_tree* t)
{
    double c[3], r;
    node_center_radius(t, 0, c, &r);
    return r;
}

/* MLoD projection of nq queries, n_iter iterations each (Fastapss::project /
 * APSSOctree::projectCPU with fast=true).  step_max < 0 selects the root box
 * radius (Fastapss.cu:448-449, CPUUtils.cpp:626-627).  visited (optional)
 * receives per query the node visits summed over iterations. */
void orc_project_mlod(const orc_tree* t, const float* q, int64_t nq, int n_iter, int ktype, double sigma,
                      double exponent, double shift, const double* sigmas, int nsig, int rule, double cutoff,
                      int min_depth, double step_max, double* out_p, double* out_n, int64_t* visited)
{
    orc_kernel k;
    kernel_from_args(&k, ktype, sigma, exponent, shift, sigmas, nsig);
    if (step_max < 0) step_max = orc_tree_radius(t);
    double thr = rule == ORC_RULE_GPU ? 1e-6 : 1e-12;
    int zero_safe = rule == ORC_RULE_GPU;
#pragma omp parallel for schedule(dynamic, 64)
    for (int64_t i = 0; i < nq; ++i) {
        mlod_ctx cx;
        cx.t = t;
        cx.k = &k;
        cx.rule = rule;
        cx.cutoff = cutoff;
        cx.min_depth = min_depth;
        cx.visited = 0;
        double cur[3] = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};
        double nrm[3] = {0, 0, 0};
        for (int it = 0; it < n_iter; ++it) {
            double acc[9] = {0};
            memcpy(cx.q, cur, sizeof cur);
            mlod_rec(&cx, 0, acc);
            double x[3];
            fit_and_project(acc, thr, zero_safe, step_max, x, nrm);
            for (int a = 0; a < 3; ++a) cur[a] += x[a];
        }
        for (int a = 0; a < 3; ++a) {
            out_p[3 * i + a] = cur[a];
            out_n[3 * i + a] = nrm[a];
        }
        if (visited) visited[i] = cx.visited;
    }
}

/* Global APSS: every point contributes (APSSOctree::APSSStats, CPUUtils.cpp:515-528;
 * GlobalAPSS.cu:113-168).  Degenerate threshold 1e-12 as both reference paths. */
void orc_project_global(const orc_tree* t, const float* q, int64_t nq, int n_iter, int ktype, double sigma,
                        double exponent, double shift, const double* sigmas, int nsig, double step_max,
                        double* out_p, double* out_n)
{
    orc_kernel k;
    kernel_from_args(&k, ktype, sigma, exponent, shift, sigmas, nsig);
    if (step_max < 0) step_max = orc_tree_radius(t);
#pragma omp parallel for schedule(dynamic, 16)
    for (int64_t i = 0; i < nq; ++i) {
        double cur[3] = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};
        double nrm[3] = {0, 0, 0};
        for (int it = 0; it < n_iter; ++it) {
            double acc[9] = {0};
            for (int64_t j = 0; j < t->n_pts; ++j) {
                double p[3] = {t->pts[3 * j], t->pts[3 * j + 1], t->pts[3 * j + 2]};
                add_point(acc, t, (int32_t)j, cur, kernel_w(&k, wdist2(p, cur), ORC_RULE_CPU));
            }
            double x[3];
            fit_and_project(acc, 1e-12, 0, step_max, x, nrm);
            for (int a = 0; a < 3; ++a) cur[a] += x[a];
        }
        for (int a = 0; a < 3; ++a) {
            out_p[3 * i + a] = cur[a];
            out_n[3 * i + a] = nrm[a];
        }
    }
}

/* ---------------------------------------------------------------- kNN / ball */

/* Squared distance exactly as kdTreeNN.h:424 evaluates it: float differences,
 * float products and float sums (no contraction), widened to double. */
static inline double kd_sqr_dist(const float* p, const float* q)
{
    volatile float dx = p[0] - q[0], dy = p[1] - q[1], dz = p[2] - q[2];
    volatile float xx = dx * dx, yy = dy * dy, zz = dz * dz;
    volatile float s = xx + yy;
    float s2 = s + zz;
    return (double)s2;
}

typedef struct {
    double d;
    int32_t i;
} dist_idx;

static int cmp_dist_idx(const void* a, const void* b)
{
    const dist_idx* x = (const dist_idx*)a;
    const dist_idx* y = (const dist_idx*)b;
    if (x->d < y->d) return -1;
    if (x->d > y->d) return 1;
    return (x->i > y->i) - (x->i < y->i);
}

/* Exact k nearest neighbours by brute force, sorted by (distance, index).
 * tie_flag[i] = 1 when the k-th and (k+1)-th distances are equal. */
void orc_knn(const float* pts, int64_t n, const float* q, int64_t nq, int k, int32_t* out_idx, double* out_d2,
             int32_t* tie_flag)
{
#pragma omp parallel
    {
        dist_idx* buf = (dist_idx*)malloc((size_t)n * sizeof(dist_idx));
#pragma omp for schedule(dynamic, 8)
        for (int64_t i = 0; i < nq; ++i) {
            for (int64_t j = 0; j < n; ++j) {
                buf[j].d = kd_sqr_dist(pts + 3 * j, q + 3 * i);
                buf[j].i = (int32_t)j;
            }
            qsort(buf, (size_t)n, sizeof(dist_idx), cmp_dist_idx);
            int kk = k < n ? k : (int)n;
            for (int j = 0; j < kk; ++j) {
                out_idx[i * k + j] = buf[j].i;
                out_d2[i * k + j] = buf[j].d;
            }
            if (tie_flag) tie_flag[i] = (kk < n && buf[kk].d == buf[kk - 1].d) ? 1 : 0;
        }
        free(buf);
    }
}

/* kNN (mode 0) or ball (mode 1) APSS, APSSOctree::projectAPSSCPU (CPUUtils.cpp:690-737):
 * raw point positions/normals, no area weights, CPU threshold 1e-12.  The query
 * position used for the gather and the weights is the current iterate rounded
 * to float, as the reference keeps it in a glm::vec3.  ball_r < 0 uses
 * 3 sigmas[0].  An empty ball returns the starting point with a zero normal. */
void orc_project_apss(const float* pts, const float* nrm, int64_t n, const float* q, int64_t nq, int n_iter,
                      int mode, int k, double ball_r, int ktype, double sigma, double exponent, double shift,
                      const double* sigmas, int nsig, double step_max, double* out_p, double* out_n)
{
    orc_kernel kk;
    kernel_from_args(&kk, ktype, sigma, exponent, shift, sigmas, nsig);
    double r = ball_r < 0 ? 3.0 * (double)(float)sigmas[0] : ball_r;
#pragma omp parallel
    {
        dist_idx* buf = (dist_idx*)malloc((size_t)n * sizeof(dist_idx));
#pragma omp for schedule(dynamic, 8)
        for (int64_t i = 0; i < nq; ++i) {
            double cur[3] = {q[3 * i], q[3 * i + 1], q[3 * i + 2]};
            double nv[3] = {0, 0, 0};
            int failed = 0;
            for (int it = 0; it < n_iter && !failed; ++it) {
                float cf[3] = {(float)cur[0], (float)cur[1], (float)cur[2]};
                int64_t m = 0;
                for (int64_t j = 0; j < n; ++j) {
                    double d = kd_sqr_dist(pts + 3 * j, cf);
                    if (mode == 1 && d > r * r) continue;
                    buf[m].d = d;
                    buf[m].i = (int32_t)j;
                    ++m;
                }
                if (mode == 0) {
                    qsort(buf, (size_t)m, sizeof(dist_idx), cmp_dist_idx);
                    if (m > k) m = k;
                } else if (m == 0) {
                    failed = 1;
                    break;
                }
                double acc[9] = {0};
                double qd[3] = {cf[0], cf[1], cf[2]};
                for (int64_t j = 0; j < m; ++j) {
                    int32_t pi = buf[j].i;
                    double p[3] = {pts[3 * pi], pts[3 * pi + 1], pts[3 * pi + 2]};
                    double w = kernel_w(&kk, wdist2(p, qd), ORC_RULE_CPU);
                    double mm[9] = {1.0, p[0], p[1], p[2], nrm[3 * pi], nrm[3 * pi + 1], nrm[3 * pi + 2], 0.0, 0.0};
                    add_moments(acc, mm, qd, w);
                }
                double x[3];
                fit_and_project(acc, 1e-12, 0, step_max, x, nv);
                for (int a = 0; a < 3; ++a) cur[a] = qd[a] + x[a];
            }
            if (failed) {
                for (int a = 0; a < 3; ++a) {
                    cur[a] = q[3 * i + a];
                    nv[a] = 0.0;
                }
            }
            for (int a = 0; a < 3; ++a) {
                out_p[3 * i + a] = cur[a];
                out_n[3 * i + a] = nv[a];
            }
        }
        free(buf);
    }
}

/* ---------------------------------------------------------------- dual contouring */

/* Corner field of scene.cpp:1388-1394: f = (c - x).n, NaN when |n|^2 < 0.5. */
void orc_dc_field(const double* corners, const double* proj, const double* nrm, int64_t n, double* f)
{
    for (int64_t i = 0; i < n; ++i) {
        const double* c = corners + 3 * i;
        const double* x = proj + 3 * i;
        const double* v = nrm + 3 * i;
        double l2 = v[0] * v[0] + v[1] * v[1] + v[2] * v[2];
        if (l2 < 0.5)
            f[i] = NAN;
        else
            f[i] = (c[0] - x[0]) * v[0] + (c[1] - x[1]) * v[1] + (c[2] - x[2]) * v[2];
    }
}

/* DC vertex of one cell from its 8 corner values (dual_contouring.h:124-176)
 * with the zero normal field the reference passes (scene.cpp:1355-1358): the
 * QEF has A = 0, so the min-norm solve returns the mass point of the edge
 * crossings; no crossing gives the cell centre.  Corner c of the cell sits at
 * lo + (c&1, c>>1&1, c>>2&1) * width.  A NaN corner compares as non-negative,
 * exactly as `(val < 0)` does in the reference. */
void orc_dc_vertex(const double* lo, double width, const double* val8, double* out, int32_t* n_cross)
{
    static const int edges[12][2] = {{0, 1}, {0, 2}, {1, 3}, {2, 3}, {4, 5}, {4, 6},
                                     {5, 7}, {6, 7}, {0, 4}, {1, 5}, {2, 6}, {3, 7}};
    double sum[3] = {0, 0, 0};
    int cnt = 0;
    for (int e = 0; e < 12; ++e) {
        int a = edges[e][0], b = edges[e][1];
        double fa = val8[a], fb = val8[b];
        if ((fa < 0) == (fb < 0)) continue;
        double x = -fa / (fb - fa);
        for (int k = 0; k < 3; ++k) {
            double ua = lo[k] + width * ((a >> k) & 1);
            double ub = lo[k] + width * ((b >> k) & 1);
            sum[k] += x * ub + (1.0 - x) * ua;
        }
        ++cnt;
    }
    if (cnt > 0) {
        for (int k = 0; k < 3; ++k) out[k] = sum[k] / cnt;
    } else {
        for (int k = 0; k < 3; ++k) out[k] = lo[k] + 0.5 * width;
    }
    if (isnan(out[0]) || isnan(out[1]) || isnan(out[2]))
        for (int k = 0; k < 3; ++k) out[k] = lo[k] + 0.5 * width;
    *n_cross = cnt;
}
