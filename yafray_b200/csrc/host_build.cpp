// Host-side SAH kd-tree build and object tree, producing the device format.
//
// The kd-tree must come out node-for-node identical to YafRay's kdTree_t
// (kdtree.cc:57-582, triclip.cc:50-240): leaf order decides which of two
// equally distant triangles a ray reports (Intersect keeps the first one it
// tests, kdtree.cc:684-714), and identical trees make the per-ray node and
// triangle counts comparable with the reference traversal.  So the split
// search, the classification order, the clipping arithmetic and the float /
// double types of every intermediate follow the reference; the code
// structure (vectors per node instead of the shared scratch arrays, an
// explicit node list instead of a growing pointer array) is our own.
//
// The reference ships built with -O3 -ffast-math (linux-settings.py:21-26),
// and g++ rewrites four expressions of the split search under that flag.
// The tree of the shipped build is the one to match, so these four are
// written here in the rewritten form (each place is marked "fast-math"):
//   1/(dx*dy + dx*dz + dy*dz)       -> 1/((dy + dz)*dx + dy*dz)
//   l / d[axis] in the binned search -> l * (1/d[axis])
//   raw - (0.1 + l/d)*eb*raw         -> raw * (1 - (l/d + 0.1)*eb)
//   lo - 0.021*h - 1e-5*s            -> lo - (0.021*h + 1e-5*s)   (and hi + ...)
#include "host_build.h"
#include "kd_clip.h"
#include "kd_sort.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <atomic>
#include <list>
#include <thread>

namespace yr {
namespace {

constexpr int kBins = 1024;          // KD_BINS (kdtree.cc:17)
constexpr uint32_t kClipThresh = 32;  // TRI_CLIP_THRESH (kdtree.cc:16)
constexpr uint32_t kPigeonThresh = 128;

// 3-way min / max with the reference's comparison order (kdtree.cc:19-20).
inline float min3(float a, float b, float c) { return (a > b) ? ((b > c) ? c : b) : ((a > c) ? c : a); }
inline float max3(float a, float b, float c) { return (a < b) ? ((b > c) ? b : c) : ((a > c) ? a : c); }

struct Bin {
    int n = 0, c_left = 0, c_right = 0, c_bleft = 0, c_both = 0;
    float t = 0.f;
    bool empty() const { return n == 0; }
};

enum EdgeEnd { kLower = 0, kBoth = 1, kUpper = 2 };  // kdtree.cc:10-12

using Edge = KdEdge;  // boundEdge (kdtree.h:64-76)

struct Split {
    int axis = -1;
    int offset = -1;
    float best_cost = 0.f;
    float old_cost = 0.f;
    float t = 0.f;
    uint32_t n_below = 0, n_above = 0;
    int n_edge = 0;
};

// Sutherland-Hodgman clip (kd_clip.h).  Returns 0 = clipped bound in
// `box`, 1 = nothing left, 2 = polygon overflow (caller keeps the full bound).
int clip_triangle(const double bmin[3], const double bmax[3], const double v[3][3], Box &box) {
    return kd_clip_triangle(bmin, bmax, v, box.a, box.g);
}

class Builder {
  public:
    Builder(const float *verts, const uint32_t *tris, uint32_t ntris, KdTree &out)
        : verts_(verts), tris_(tris), n_(ntris), out_(out) {}

    // a builder for one deferred subtree, sharing the parent's inputs
    Builder(const Builder &parent, KdTree &out)
        : verts_(parent.verts_), tris_(parent.tris_), n_(parent.n_), out_(out), shared_bounds_(&parent.bounds()),
          tree_(parent.tree_), cost_ratio_(parent.cost_ratio_), ebonus_(parent.ebonus_),
          max_depth_(parent.max_depth_), max_leaf_(parent.max_leaf_) {}

    struct Task {
        std::vector<uint32_t> prims;
        Box nb;
        int depth;
        int bad_refines;
        size_t node;  // placeholder position in the parent's node array
    };

    yr_status run(const KdParams &kp, int nthreads) {
        // kdTree_t ctor parameter defaults (kdtree.cc:57-80)
        ebonus_ = kp.empty_bonus;
        kd_limits(n_, kp, max_depth_, max_leaf_, cost_ratio_);
        if (nthreads > 1 && n_ > 4096) {
            defer_depth_ = 0;
            while ((1 << defer_depth_) < 4 * nthreads && defer_depth_ < 12) defer_depth_++;
        }

        bounds_.resize(n_);
        for (uint32_t i = 0; i < n_; i++) {
            const float *A = vtx(i, 0), *B = vtx(i, 1), *C = vtx(i, 2);
            Box &b = bounds_[i];
            for (int k = 0; k < 3; k++) {
                b.a[k] = min3(A[k], B[k], C[k]);
                b.g[k] = max3(A[k], B[k], C[k]);
            }
            if (i == 0) {
                tree_ = b;
            } else {
                // bound_t(const bound_t&, const bound_t&) with MIN/MAX (bound.cc:32-52)
                for (int k = 0; k < 3; k++) {
                    tree_.a[k] = (tree_.a[k] < b.a[k]) ? tree_.a[k] : b.a[k];
                    tree_.g[k] = (tree_.g[k] > b.g[k]) ? tree_.g[k] : b.g[k];
                }
            }
        }
        tree_ = kd_grow_bound(tree_);
        std::vector<uint32_t> all(n_);
        for (uint32_t i = 0; i < n_; i++) all[i] = i;
        out_.nodes.clear();
        out_.prims.clear();
        out_.nodes.reserve(2 * (size_t)n_ + 16);
        Box root = tree_;
        yr_status st = build(all, root, 0, 0);
        if (st == YR_OK && !tasks_.empty()) st = run_tasks(nthreads);
        out_.bound = tree_;
        out_.max_depth = max_depth_;
        out_.max_leaf_size = max_leaf_;
        out_.cost_ratio = cost_ratio_;
        out_.empty_bonus = ebonus_;
        return st;
    }

    const std::vector<Box> &bounds() const { return shared_bounds_ ? *shared_bounds_ : bounds_; }

    // kdTree_t::buildTree (kdtree.cc:416-582)
    yr_status build(std::vector<uint32_t> &prims, const Box &nb, int depth, int bad_refines);

  private:
    const float *vtx(uint32_t tri, int k) const { return verts_ + 3 * (size_t)tris_[3 * (size_t)tri + k]; }

    // Build the deferred subtrees in parallel and splice each one in place of
    // its placeholder: the node order is then the sequential build's
    // depth-first order (right-child links and prim offsets relocated).
    yr_status run_tasks(int nthreads) {
        std::vector<KdTree> sub(tasks_.size());
        std::vector<yr_status> st(tasks_.size(), YR_OK);
        std::atomic<size_t> next{0};
        auto worker = [&] {
            for (;;) {
                const size_t k = next.fetch_add(1);
                if (k >= tasks_.size()) return;
                Builder b(*this, sub[k]);
                Task &t = tasks_[k];
                try {
                    st[k] = b.build(t.prims, t.nb, t.depth, t.bad_refines);
                } catch (const std::bad_alloc &) {
                    st[k] = YR_ERR_OUT_OF_MEMORY;
                }
            }
        };
        std::vector<std::thread> pool;
        for (int i = 1; i < nthreads; i++) pool.emplace_back(worker);
        worker();
        for (std::thread &th : pool) th.join();
        for (yr_status e : st)
            if (e != YR_OK) return e;
        // new position of every node of the serial part
        const size_t n0 = out_.nodes.size();
        std::vector<size_t> newpos(n0 + 1);
        std::vector<int> task_at(n0, -1);
        for (size_t k = 0; k < tasks_.size(); k++) task_at[tasks_[k].node] = (int)k;
        size_t shift = 0;
        for (size_t i = 0; i < n0; i++) {
            newpos[i] = i + shift;
            if (task_at[i] >= 0) shift += sub[task_at[i]].nodes.size() - 1;
        }
        newpos[n0] = n0 + shift;
        if (n0 + shift >= (1u << 30)) return YR_ERR_TOO_LARGE;
        std::vector<yr_kd_node> nodes(n0 + shift);
        std::vector<uint32_t> prims = std::move(out_.prims);
        for (size_t i = 0; i < n0; i++) {
            const yr_kd_node nd = out_.nodes[i];
            const int k = task_at[i];
            if (k < 0) {
                yr_kd_node o = nd;
                if ((nd.flags & 3u) != 3u) o.flags = (nd.flags & 3u) | ((uint32_t)newpos[nd.flags >> 2] << 2);
                nodes[newpos[i]] = o;
                continue;
            }
            const KdTree &t = sub[k];
            const uint32_t base = (uint32_t)newpos[i], pbase = (uint32_t)prims.size();
            for (size_t j = 0; j < t.nodes.size(); j++) {
                yr_kd_node o = t.nodes[j];
                if ((o.flags & 3u) != 3u) o.flags = (o.flags & 3u) | (((o.flags >> 2) + base) << 2);
                else if ((o.flags >> 2) > 1) o.word += pbase;
                nodes[base + j] = o;
            }
            prims.insert(prims.end(), t.prims.begin(), t.prims.end());
        }
        out_.nodes.swap(nodes);
        out_.prims.swap(prims);
        return YR_OK;
    }

    void make_leaf(const std::vector<uint32_t> &prims) {
        yr_kd_node nd;
        const uint32_t np = (uint32_t)prims.size();
        nd.flags = (np << 2) | 3u;
        if (np == 1) {
            nd.word = prims[0];
        } else if (np > 1) {
            nd.word = (uint32_t)out_.prims.size();
            out_.prims.insert(out_.prims.end(), prims.begin(), prims.end());
        } else {
            nd.word = 0;
        }
        out_.nodes.push_back(nd);
    }

    // Binned SAH for > 128 primitives (kdTree_t::pigeonMinCost, kdtree.cc:167-304).
    yr_status pigeon(const std::vector<uint32_t> &prims, const Box &nb, float ebonus, Split &sp) {
        const uint32_t np = (uint32_t)prims.size();
        float d[3] = {nb.g[0] - nb.a[0], nb.g[1] - nb.a[1], nb.g[2] - nb.a[2]};
        sp.old_cost = float(np);
        sp.best_cost = std::numeric_limits<float>::infinity();
        const float inv_sa = 1.0f / ((d[1] + d[2]) * d[0] + d[1] * d[2]);  // fast-math
        std::vector<Bin> bin(kBins + 1);
        for (int axis = 0; axis < 3; axis++) {
            const float s = kBins / d[axis];
            const float lo = nb.a[axis];
            for (uint32_t i = 0; i < np; i++) {
                const Box &bb = bounds()[prims[i]];
                const float tl = bb.a[axis], tu = bb.g[axis];
                int bl = (int)((tl - lo) * s), br = (int)((tu - lo) * s);
                bl = bl < 0 ? 0 : (bl > kBins ? kBins : bl);
                br = br < 0 ? 0 : (br > kBins ? kBins : br);
                Bin &L = bin[bl];
                if (tl == tu) {
                    if (L.empty() || tl >= L.t) {
                        L.t = tl;
                        L.c_both++;
                    } else {
                        L.c_left++;
                        L.c_right++;
                    }
                    L.n += 2;
                } else {
                    if (L.empty() || tl > L.t) {
                        L.t = tl;
                        L.c_left += L.c_both + L.c_bleft;
                        L.c_right += L.c_both;
                        L.c_both = L.c_bleft = 0;
                        L.c_bleft++;
                    } else if (tl == L.t) {
                        L.c_bleft++;
                    } else {
                        L.c_left++;
                    }
                    L.n++;
                    Bin &R = bin[br];
                    R.c_right++;
                    if (R.empty() || tu > R.t) {
                        R.t = tu;
                        R.c_left += R.c_both + R.c_bleft;
                        R.c_right += R.c_both;
                        R.c_both = R.c_bleft = 0;
                    }
                    R.n++;
                }
            }
            const float cap_area = d[(axis + 1) % 3] * d[(axis + 2) % 3];
            const float cap_perim = d[(axis + 1) % 3] + d[(axis + 2) % 3];
            const float rd = 1.0f / d[axis];  // fast-math: reciprocal hoisted out of the loop
            uint32_t below = 0, above = np;
            for (int i = 0; i <= kBins; i++) {
                const Bin &b = bin[i];
                if (b.empty()) continue;
                below += b.c_left;
                above -= b.c_right;
                const float et = b.t;
                if (et > nb.a[axis] && et < nb.g[axis]) {
                    const float l1 = et - nb.a[axis], l2 = nb.g[axis] - et;
                    const float below_sa = cap_area + l1 * cap_perim;
                    const float above_sa = cap_area + l2 * cap_perim;
                    const float raw = below_sa * below + above_sa * above;
                    // fast-math: raw - (0.1 + l*rd)*eb*raw folded to raw*(1 - (l*rd + 0.1)*eb)
                    float net;
                    if (above == 0) net = raw * (1.0f - (l2 * rd + 0.1f) * ebonus);
                    else if (below == 0) net = raw * (1.0f - (l1 * rd + 0.1f) * ebonus);
                    else net = raw;
                    const float cost = cost_ratio_ + inv_sa * net;
                    if (cost < sp.best_cost) {
                        sp.t = et;
                        sp.best_cost = cost;
                        sp.axis = axis;
                        sp.offset = i;
                        sp.n_below = below;
                        sp.n_above = above;
                    }
                }
                below += b.c_both + b.c_bleft;
                above -= b.c_both;
            }
            // the reference prints "SCREWED!!" and exits here (kdtree.cc:283-301)
            if (below != np || above != 0) return YR_ERR_BAD_TREE;
            std::fill(bin.begin(), bin.end(), Bin());
        }
        return YR_OK;
    }

    // Exact sorted-edge SAH (kdTree_t::minimalCost, kdtree.cc:311-406).
    // `clipped` holds per-position bounds (after clipping), else bounds()[prim].
    void exact(const std::vector<uint32_t> &prims, const Box &nb, const std::vector<Box> *clipped,
               float ebonus, Split &sp) {
        const uint32_t np = (uint32_t)prims.size();
        float d[3] = {nb.g[0] - nb.a[0], nb.g[1] - nb.a[1], nb.g[2] - nb.a[2]};
        sp.old_cost = float(np);
        sp.best_cost = std::numeric_limits<float>::infinity();
        const float inv_sa = 1.0f / ((d[1] + d[2]) * d[0] + d[1] * d[2]);  // fast-math
        for (int axis = 0; axis < 3; axis++) {
            std::vector<Edge> &ed = edges_[axis];
            ed.clear();
            for (uint32_t i = 0; i < np; i++) {
                const int pn = (int)prims[i];
                const Box &bb = clipped ? (*clipped)[i] : bounds()[pn];
                if (bb.a[axis] == bb.g[axis]) {
                    ed.push_back({bb.a[axis], pn, kBoth});
                } else {
                    ed.push_back({bb.a[axis], pn, kLower});
                    ed.push_back({bb.g[axis], pn, kUpper});
                }
            }
            kd_sort(ed.data(), (int)ed.size());  // std::sort's permutation (kd_sort.h)
            const int ne = (int)ed.size();
            const float cap_area = d[(axis + 1) % 3] * d[(axis + 2) % 3];
            const float cap_perim = d[(axis + 1) % 3] + d[(axis + 2) % 3];
            uint32_t below = 0, above = np;
            for (int i = 0; i < ne; ++i) {
                if (ed[i].end == kUpper) --above;
                const float et = ed[i].pos;
                if (et > nb.a[axis] && et < nb.g[axis]) {
                    const float l1 = et - nb.a[axis], l2 = nb.g[axis] - et;
                    const float below_sa = cap_area + l1 * cap_perim;
                    const float above_sa = cap_area + l2 * cap_perim;
                    const float raw = below_sa * below + above_sa * above;
                    // fast-math: folded as in the binned search, division kept here
                    float net;
                    if (above == 0) net = raw * (1.0f - (l2 / d[axis] + 0.1f) * ebonus);
                    else if (below == 0) net = raw * (1.0f - (l1 / d[axis] + 0.1f) * ebonus);
                    else net = raw;
                    const float cost = cost_ratio_ + inv_sa * net;
                    if (cost < sp.best_cost) {
                        sp.best_cost = cost;
                        sp.axis = axis;
                        sp.offset = i;
                        sp.n_edge = ne;
                        sp.n_below = below;
                        sp.n_above = above;
                    }
                }
                if (ed[i].end != kUpper) {
                    ++below;
                    if (ed[i].end == kBoth) --above;
                }
            }
        }
    }

  public:
    yr_status build_node(std::vector<uint32_t> &prims, const Box &nb, int depth, int bad_refines) {
        if (defer_depth_ >= 0 && depth == defer_depth_ && prims.size() > 4096) {
            Task t;
            t.prims.swap(prims);
            t.nb = nb;
            t.depth = depth;
            t.bad_refines = bad_refines;
            t.node = out_.nodes.size();
            tasks_.push_back(std::move(t));
            out_.nodes.push_back(yr_kd_node{0u, 3u});  // placeholder
            return YR_OK;
        }
        std::vector<Box> clipped;
        if (prims.size() <= kClipThresh) {
            double bmin[3], bmax[3];
            for (int i = 0; i < 3; ++i) {
                const double half = (double)nb.g[i] - (double)nb.a[i];
                const double tsize = (double)tree_.g[i] - (double)tree_.a[i];
                const double grow = 0.021 * half + 0.00001 * tsize;  // fast-math
                bmin[i] = (double)nb.a[i] - grow;
                bmax[i] = (double)nb.g[i] + grow;
            }
            std::vector<uint32_t> kept;
            kept.reserve(prims.size());
            clipped.reserve(prims.size());
            for (uint32_t pn : prims) {
                double v[3][3];
                for (int j = 0; j < 3; ++j) {
                    v[0][j] = vtx(pn, 0)[j];
                    v[1][j] = vtx(pn, 1)[j];
                    v[2][j] = vtx(pn, 2)[j];
                }
                Box cb;
                int res = clip_triangle(bmin, bmax, v, cb);
                if (res == 0) {
                    kept.push_back(pn);
                    clipped.push_back(cb);
                } else if (res == 2) {
                    kept.push_back(pn);
                    clipped.push_back(bounds()[pn]);
                }
            }
            prims.swap(kept);
        }
        const uint32_t np = (uint32_t)prims.size();
        if (np <= (uint32_t)max_leaf_ || depth >= max_depth_) {
            make_leaf(prims);
            return YR_OK;
        }
        Split sp;
        const float eb = (float)(ebonus_ * (1.1 - (double)((float)depth / (float)max_depth_)));
        if (np > kPigeonThresh) {
            yr_status st = pigeon(prims, nb, eb, sp);
            if (st != YR_OK) return st;
        } else if (np > kClipThresh) {
            exact(prims, nb, nullptr, eb, sp);
        } else {
            exact(prims, nb, &clipped, eb, sp);
        }
        if (sp.best_cost > sp.old_cost) ++bad_refines;
        if ((sp.best_cost > 1.6f * sp.old_cost && np < 16) || sp.axis == -1 || bad_refines == 2) {
            make_leaf(prims);
            return YR_OK;
        }
        std::vector<uint32_t> left, right;
        left.reserve(np);
        right.reserve(np);
        float split_pos;
        const int ax = sp.axis;
        if (np > kPigeonThresh) {
            for (uint32_t pn : prims) {
                if (bounds()[pn].a[ax] >= sp.t) {
                    right.push_back(pn);
                } else {
                    left.push_back(pn);
                    if (bounds()[pn].g[ax] > sp.t) right.push_back(pn);
                }
            }
            split_pos = sp.t;
        } else {
            const std::vector<Edge> &ed = edges_[ax];
            split_pos = ed[sp.offset].pos;
            for (int i = 0; i < sp.offset; ++i)
                if (ed[i].end != kUpper) left.push_back((uint32_t)ed[i].prim);
            if (ed[sp.offset].end == kBoth) right.push_back((uint32_t)ed[sp.offset].prim);
            for (int i = sp.offset + 1; i < sp.n_edge; ++i)
                if (ed[i].end != kLower) right.push_back((uint32_t)ed[i].prim);
        }
        prims.clear();
        prims.shrink_to_fit();
        clipped.clear();
        clipped.shrink_to_fit();

        const size_t cur = out_.nodes.size();
        yr_kd_node nd;
        std::memcpy(&nd.word, &split_pos, 4);
        nd.flags = (uint32_t)ax;
        out_.nodes.push_back(nd);
        Box bl = nb, br = nb;
        bl.g[ax] = split_pos;
        br.a[ax] = split_pos;
        yr_status st = build_node(left, bl, depth + 1, bad_refines);
        if (st != YR_OK) return st;
        const size_t right_index = out_.nodes.size();
        if (right_index >= (1u << 30)) return YR_ERR_TOO_LARGE;
        out_.nodes[cur].flags = (out_.nodes[cur].flags & 3u) | ((uint32_t)right_index << 2);
        return build_node(right, br, depth + 1, bad_refines);
    }
  private:

    const float *verts_;
    const uint32_t *tris_;
    uint32_t n_;
    KdTree &out_;
    std::vector<Box> bounds_;
    const std::vector<Box> *shared_bounds_ = nullptr;
    Box tree_{};
    float cost_ratio_ = 0.f, ebonus_ = 0.f;
    int max_depth_ = 0, max_leaf_ = 0;
    int defer_depth_ = -1;
    std::vector<Task> tasks_;
    std::vector<Edge> edges_[3];
};

yr_status Builder::build(std::vector<uint32_t> &prims, const Box &nb, int depth, int bad_refines) {
    return build_node(prims, nb, depth, bad_refines);
}

// --- object tree -----------------------------------------------------------

float box_vol(const Box &b) { return (b.g[1] - b.a[1]) * (b.g[0] - b.a[0]) * (b.g[2] - b.a[2]); }

Box box_union(const Box &r, const Box &l) {
    Box o;
    for (int k = 0; k < 3; k++) {
        o.a[k] = (r.a[k] < l.a[k]) ? r.a[k] : l.a[k];
        o.g[k] = (r.g[k] > l.g[k]) ? r.g[k] : l.g[k];
    }
    return o;
}

// b_intersect + bound_distance (bound.cc:61-83)
float box_overlap(const Box &r, const Box &l) {
    float minx = (r.a[0] > l.a[0]) ? r.a[0] : l.a[0];
    float miny = (r.a[1] > l.a[1]) ? r.a[1] : l.a[1];
    float minz = (r.a[2] > l.a[2]) ? r.a[2] : l.a[2];
    float maxx = (r.g[0] < l.g[0]) ? r.g[0] : l.g[0];
    float maxy = (r.g[1] < l.g[1]) ? r.g[1] : l.g[1];
    float maxz = (r.g[2] < l.g[2]) ? r.g[2] : l.g[2];
    if (maxx <= minx) return 0;
    if (maxy <= miny) return 0;
    if (maxz <= minz) return 0;
    return (maxx - minx) * (maxy - miny) * (maxz - minz);
}

float box_distance(const Box &l, const Box &r) {
    Box nb = box_union(l, r);
    float voids = box_vol(nb) - box_vol(l) - box_vol(r) + box_overlap(l, r);
    if (voids < 0) voids = 0;
    return (float)((double)(voids + box_vol(nb)) + std::fabs((double)(box_vol(l) - box_vol(r))));
}

// Greedy nearest-pair clustering with lazily recomputed nearest neighbours
// (treeBuilder_t, yafutils.h:10-190).  The neighbour bookkeeping decides
// which pair merges first when distances tie, so it is kept as is.
class Clusterer {
  public:
    explicit Clusterer(std::vector<ObjNode> &nodes, std::vector<Box> &boxes) : nodes_(nodes), boxes_(boxes) {}

    void push(int obj) {
        items_.push_front(Item(obj));
        items_.front().nearest = items_.end();
        calculate(items_.begin());
        if (items_.size() > 1 && (items_.front().dist < mindist_ || best_ == items_.end())) {
            best_ = items_.begin();
            mindist_ = items_.begin()->dist;
        }
    }

    void build() {
        while (items_.size() >= 2) step();
    }

    int solution() const { return items_.front().obj; }

  private:
    struct Item;
    using It = std::list<Item>::iterator;
    struct Item {
        explicit Item(int o) : obj(o) {}
        int obj;
        It nearest;
        float dist = 0.f;
        std::list<It> recalculate;
    };

    float distance(int a, int b) const { return box_distance(boxes_[a], boxes_[b]); }

    void calculate(It n) {
        if (items_.size() == 1) return;
        if (items_.size() == 2) {
            It a = items_.begin();
            It b = a;
            ++b;
            a->nearest = b;
            a->recalculate.push_back(b);
            b->nearest = a;
            b->recalculate.push_back(a);
            mindist_ = a->dist = b->dist = distance(a->obj, b->obj);
            best_ = a;
            return;
        }
        It before = n->nearest;
        Item &nu = *n;
        for (It i = items_.begin(); i != items_.end(); ++i) {
            if (i == n) continue;
            float d = distance(nu.obj, i->obj);
            if (i->nearest == items_.end()) {
                i->nearest = n;
                i->dist = d;
                nu.recalculate.push_back(i);
            }
            bool old_useless = (nu.nearest == items_.end()) || (nu.nearest->dist < nu.dist);
            bool new_useful = (d < i->dist);
            if ((nu.nearest == items_.end()) || ((d < nu.dist) && (new_useful || old_useless)) ||
                (old_useless && new_useful)) {
                nu.nearest = i;
                nu.dist = d;
            }
        }
        if (nu.dist < nu.nearest->dist) {
            nu.nearest->nearest->recalculate.remove(nu.nearest);
            nu.nearest->nearest = n;
            nu.nearest->dist = nu.dist;
            nu.recalculate.push_back(nu.nearest);
        }
        if (before != items_.end()) before->recalculate.remove(n);
        nu.nearest->recalculate.push_back(n);
    }

    void pop() {
        best_->nearest->nearest->recalculate.remove(best_->nearest);
        std::list<It> update = best_->recalculate;
        best_->nearest->recalculate.remove(best_);
        update.insert(update.end(), best_->nearest->recalculate.begin(), best_->nearest->recalculate.end());
        items_.erase(best_->nearest);
        items_.erase(best_);
        if (!items_.empty()) {
            best_ = items_.end();
            for (It i : update) i->nearest = items_.end();
            for (It i : update) calculate(i);
            for (It i = items_.begin(); i != items_.end(); ++i)
                if ((i->dist < mindist_) || (best_ == items_.end())) {
                    best_ = i;
                    mindist_ = i->dist;
                }
        }
    }

    void step() {
        const int a = best_->obj, b = best_->nearest->obj;
        // join (oTreeJoin_f, object3d.cc:22-28): left = a, right = b
        ObjNode nd;
        const Box u = box_union(boxes_[a], boxes_[b]);
        for (int k = 0; k < 3; k++) {
            nd.bmin[k] = u.a[k];
            nd.bmax[k] = u.g[k];
        }
        nd.left = a;
        nd.right = b;
        nodes_.push_back(nd);
        boxes_.push_back(u);
        pop();
        push((int)nodes_.size() - 1);
    }

    std::vector<ObjNode> &nodes_;
    std::vector<Box> &boxes_;
    std::list<Item> items_;
    It best_ = items_.end();
    float mindist_ = 0.f;
};

}  // namespace

void kd_limits(uint32_t n, const KdParams &kp, int &max_depth, int &max_leaf, float &cost_ratio) {
    cost_ratio = kp.cost_ratio;
    max_depth = kp.max_depth;
    max_leaf = kp.max_leaf;
    if (max_depth <= 0) max_depth = int(6.0f + 1.66f * std::log(float(n)));
    const double log_leaves = 1.442695f * std::log(double(n));
    if (max_leaf <= 0) {
        max_leaf = int(log_leaves - 16.0);
        if (max_leaf <= 0) max_leaf = 1;
    }
    if (max_depth > 64) max_depth = 64;
    if (kp.large_scene_penalty && log_leaves > 16.0) cost_ratio = (float)(cost_ratio + 0.25 * (log_leaves - 16.0));
}

Box kd_grow_bound(const Box &b) {
    Box t = b;
    const float dx = t.g[0] - t.a[0], dy = t.g[1] - t.a[1], dz = t.g[2] - t.a[2];
    const float diag = (float)(std::sqrt(dx * dx + dy * dy + dz * dz) * 0.0001);
    for (int k = 0; k < 3; k++) {
        t.a[k] -= diag;
        t.g[k] += diag;
    }
    return t;
}

yr_status build_kdtree(const float *verts, uint32_t nverts, const uint32_t *tris, uint32_t ntris, KdTree &out,
                       const KdParams &params, int nthreads) {
    if (!verts || !tris || ntris == 0) return YR_ERR_EMPTY_SCENE;
    for (size_t i = 0; i < 3 * (size_t)ntris; i++)
        if (tris[i] >= nverts) return YR_ERR_INVALID_ARG;
    Builder b(verts, tris, ntris, out);
    return b.run(params, nthreads);
}

Box mesh_bound(const float *verts, const uint32_t *tris, uint32_t ntris) {
    Box b;
    const float *p0 = verts + 3 * (size_t)tris[0];
    for (int k = 0; k < 3; k++) b.a[k] = b.g[k] = p0[k];
    for (size_t t = 0; t < ntris; t++)
        for (int v = 0; v < 3; v++) {
            const float *p = verts + 3 * (size_t)tris[3 * t + v];
            for (int k = 0; k < 3; k++) {
                if (p[k] > b.g[k]) b.g[k] = p[k];
                if (p[k] < b.a[k]) b.a[k] = p[k];
            }
        }
    // grown by BOX_MIN = 0.00001 (mesh.cc:32, 373-379), in double
    for (int k = 0; k < 3; k++) {
        b.a[k] = (float)((double)b.a[k] - 0.00001);
        b.g[k] = (float)((double)b.g[k] + 0.00001);
    }
    return b;
}

void build_object_tree(const std::vector<Box> &object_bounds, std::vector<ObjNode> &out) {
    // Work list: leaves first (one per object, obj_list order), then joins.
    std::vector<ObjNode> nodes;
    std::vector<Box> boxes;
    for (size_t i = 0; i < object_bounds.size(); i++) {
        ObjNode nd;
        for (int k = 0; k < 3; k++) {
            nd.bmin[k] = object_bounds[i].a[k];
            nd.bmax[k] = object_bounds[i].g[k];
        }
        nd.left = -1;
        nd.right = (int32_t)i;
        nodes.push_back(nd);
        boxes.push_back(object_bounds[i]);
    }
    out.clear();
    if (nodes.empty()) return;
    Clusterer c(nodes, boxes);
    for (size_t i = 0; i < object_bounds.size(); i++) c.push((int)i);
    c.build();
    const int root = c.solution();
    // re-index depth first from the root so that node 0 is the root
    std::vector<int> stack{root};
    std::vector<int> order;
    std::vector<int> newidx(nodes.size(), -1);
    while (!stack.empty()) {
        int n = stack.back();
        stack.pop_back();
        newidx[n] = (int)order.size();
        order.push_back(n);
        if (nodes[n].left >= 0) {
            stack.push_back(nodes[n].right);
            stack.push_back(nodes[n].left);
        }
    }
    out.resize(order.size());
    for (size_t i = 0; i < order.size(); i++) {
        ObjNode nd = nodes[order[i]];
        if (nd.left >= 0) {
            nd.left = newidx[nd.left];
            nd.right = newidx[nd.right];
        }
        out[i] = nd;
    }
}

// ------------------------------------------------------------ SAH BVH
namespace {

float half_area(const Box &b) {
    const float dx = b.g[0] - b.a[0], dy = b.g[1] - b.a[1], dz = b.g[2] - b.a[2];
    return dx * dy + dy * dz + dz * dx;
}

void grow(Box &b, const Box &c) {
    for (int k = 0; k < 3; k++) {
        b.a[k] = std::min(b.a[k], c.a[k]);
        b.g[k] = std::max(b.g[k], c.g[k]);
    }
}

Box empty_box() {
    Box b;
    for (int k = 0; k < 3; k++) {
        b.a[k] = std::numeric_limits<float>::infinity();
        b.g[k] = -std::numeric_limits<float>::infinity();
    }
    return b;
}

int sah_node(const std::vector<Box> &bb, std::vector<int> &ids, int lo, int hi, std::vector<ObjNode> &out) {
    const int me = (int)out.size();
    out.push_back(ObjNode{});
    Box all = empty_box();
    for (int i = lo; i < hi; i++) grow(all, bb[ids[i]]);
    for (int k = 0; k < 3; k++) {
        out[me].bmin[k] = all.a[k];
        out[me].bmax[k] = all.g[k];
    }
    if (hi - lo == 1) {
        out[me].left = -1;
        out[me].right = ids[lo];
        return me;
    }
    const int n = hi - lo;
    int best_axis = 0, best_split = lo + n / 2;
    double best = std::numeric_limits<double>::infinity();
    std::vector<float> right_area(n);
    for (int axis = 0; axis < 3; axis++) {
        auto centre = [&](int id) { return bb[id].a[axis] + bb[id].g[axis]; };
        std::stable_sort(ids.begin() + lo, ids.begin() + hi, [&](int x, int y) { return centre(x) < centre(y); });
        Box r = empty_box();
        for (int i = n - 1; i >= 1; i--) {
            grow(r, bb[ids[lo + i]]);
            right_area[i] = half_area(r);
        }
        Box l = empty_box();
        for (int i = 1; i < n; i++) {
            grow(l, bb[ids[lo + i - 1]]);
            const double c = (double)half_area(l) * i + (double)right_area[i] * (n - i);
            if (c < best) {
                best = c;
                best_axis = axis;
                best_split = lo + i;
            }
        }
    }
    auto centre = [&](int id) { return bb[id].a[best_axis] + bb[id].g[best_axis]; };
    std::stable_sort(ids.begin() + lo, ids.begin() + hi, [&](int x, int y) { return centre(x) < centre(y); });
    const int l = sah_node(bb, ids, lo, best_split, out);
    const int r = sah_node(bb, ids, best_split, hi, out);
    out[me].left = l;
    out[me].right = r;
    return me;
}

}  // namespace

void build_sah_object_bvh(const std::vector<Box> &object_bounds, const std::vector<int> &ids,
                          std::vector<ObjNode> &out) {
    out.clear();
    if (ids.empty()) return;
    std::vector<int> work(ids);
    out.reserve(2 * ids.size());
    sah_node(object_bounds, work, 0, (int)work.size(), out);
}

// ------------------------------------------------------------ smoothing
namespace {

struct N3 {
    float x, y, z;
};

// vector3d_t::normalize with its length summed as the caller's build sums it
N3 norm_sum_xyz(N3 a) {  // (x*x + y*y) + z*z
    const float l = a.x * a.x + a.y * a.y + a.z * a.z;
    if (l != 0.f) {
        const float k = (float)(1.0 / std::sqrt((double)l));
        a.x *= k;
        a.y *= k;
        a.z *= k;
    }
    return a;
}

N3 norm_sum_yxz(N3 a) {  // y*y + (x*x + z*z): the vertex-normal pass (fast-math)
    const float l = a.y * a.y + (a.x * a.x + a.z * a.z);
    if (l != 0.f) {
        const float k = (float)(1.0 / std::sqrt((double)l));
        a.x *= k;
        a.y *= k;
        a.z *= k;
    }
    return a;
}

}  // namespace

void smooth_normals(const float *verts, const uint32_t *tris, uint32_t nverts, uint32_t ntris, float angle,
                    std::vector<float> &corner) {
    corner.assign(9 * (size_t)ntris, 0.f);
    if (!(angle >= 1.f)) return;
    // face normals as triangle_t::setVertices forms them: (b-a)^(c-a), normalized
    std::vector<N3> fn(ntris);
    for (uint32_t t = 0; t < ntris; t++) {
        const float *a = verts + 3 * tris[3 * t], *b = verts + 3 * tris[3 * t + 1], *c = verts + 3 * tris[3 * t + 2];
        const N3 u{b[0] - a[0], b[1] - a[1], b[2] - a[2]}, v{c[0] - a[0], c[1] - a[1], c[2] - a[2]};
        fn[t] = norm_sum_xyz(N3{u.y * v.z - u.z * v.y, u.z * v.x - u.x * v.z, u.x * v.y - u.y * v.x});
    }
    if (angle >= 180.f) {  // one normal per vertex: the sum of its faces' normals
        std::vector<N3> vn(nverts, N3{0.f, 0.f, 0.f});
        for (uint32_t t = 0; t < ntris; t++)
            for (int k = 0; k < 3; k++) {
                N3 &n = vn[tris[3 * t + k]];
                n.x += fn[t].x;
                n.y += fn[t].y;
                n.z += fn[t].z;
            }
        for (N3 &n : vn) n = norm_sum_yxz(n);
        for (uint32_t t = 0; t < ntris; t++)
            for (int k = 0; k < 3; k++) {
                const N3 &n = vn[tris[3 * t + k]];
                float *o = &corner[9 * (size_t)t + 3 * k];
                o[0] = n.x;
                o[1] = n.y;
                o[2] = n.z;
            }
        return;
    }
    // per corner: the faces around the vertex whose normal is within the angle
    const float cosa = (float)std::cos((double)angle * M_PI / 180.0);
    std::vector<std::vector<uint32_t>> cnx(nverts);
    for (uint32_t t = 0; t < ntris; t++)
        for (int k = 0; k < 3; k++) cnx[tris[3 * t + k]].push_back(t);
    for (uint32_t t = 0; t < ntris; t++) {
        const N3 &N = fn[t];
        for (int k = 0; k < 3; k++) {
            N3 sn{0.f, 0.f, 0.f};
            for (uint32_t o : cnx[tris[3 * t + k]]) {
                const N3 &m = fn[o];
                const float d = m.y * N.y + (m.z * N.z + m.x * N.x);  // fast-math order of the dot
                if (cosa < d) {
                    sn.x += m.x;
                    sn.y += m.y;
                    sn.z += m.z;
                }
            }
            sn = norm_sum_xyz(sn);
            float *o = &corner[9 * (size_t)t + 3 * k];
            o[0] = sn.x;
            o[1] = sn.y;
            o[2] = sn.z;
        }
    }
}

}  // namespace yr

// ------------------------------------------------------------ instances
namespace yr {

bool instance_xf(const float *M16, InstanceXf &out) {
    // matrix4x4_t::inverse: Gauss-Jordan with partial pivoting on the
    // largest |m[k][i]|, rows divided by the pivot, then reduced
    float m[4][4], id[4][4];
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++) {
            m[i][j] = M16[4 * i + j];
            id[i][j] = i == j ? 1.0f : 0.0f;
        }
    for (int i = 0; i < 4; i++) {
        float mx = 0;
        int ci = 0;
        for (int k = i; k < 4; k++)
            if (std::fabs(m[k][i]) > mx) {
                mx = std::fabs(m[k][i]);
                ci = k;
            }
        if (mx == 0) return false;
        for (int j = 0; j < 4; j++) {
            std::swap(m[i][j], m[ci][j]);
            std::swap(id[i][j], id[ci][j]);
        }
        float f = m[i][i];
        for (int j = 0; j < 4; j++) m[i][j] /= f;
        for (int j = 0; j < 4; j++) id[i][j] /= f;
        for (int k = 0; k < 4; k++) {
            if (k == i) continue;
            f = m[k][i];
            for (int j = 0; j < 4; j++) m[k][j] -= m[i][j] * f;
            for (int j = 0; j < 4; j++) id[k][j] -= id[i][j] * f;
        }
    }
    for (int i = 0; i < 3; i++)
        for (int j = 0; j < 4; j++) {
            out.m[4 * i + j] = M16[4 * i + j];
            out.back[4 * i + j] = id[i][j];
        }
    // MRot: each row of M's 3x3 part normalised (vector3d_t::normalize)
    for (int i = 0; i < 3; i++) {
        const float x = M16[4 * i], y = M16[4 * i + 1], z = M16[4 * i + 2];
        float l = x * x + y * y + z * z;
        float k = 1.f;
        if (l != 0.f) k = (float)(1.0 / std::sqrt((double)l));
        out.rot[3 * i] = l != 0.f ? x * k : x;
        out.rot[3 * i + 1] = l != 0.f ? y * k : y;
        out.rot[3 * i + 2] = l != 0.f ? z * k : z;
    }
    return true;
}

Box instance_bound(const Box &b, const float *M) {
    // the eight corners: x and y take a or g (the shipped build folds
    // a + (g - a) to g), z takes a.z or a.z + (g.z - a.z); each placed by
    // M with its sums grouped (m0*x + m1*y) + (m2*z + m3)
    const float toz = b.g[2] - b.a[2];
    const float zs[2] = {b.a[2], b.a[2] + toz};
    Box o;
    bool first = true;
    for (int iz = 0; iz < 2; iz++)
        for (int iy = 0; iy < 2; iy++)
            for (int ix = 0; ix < 2; ix++) {
                const float x = ix ? b.g[0] : b.a[0], y = iy ? b.g[1] : b.a[1], z = zs[iz];
                float p[3];
                for (int r = 0; r < 3; r++)
                    p[r] = (M[4 * r] * x + M[4 * r + 1] * y) + (M[4 * r + 2] * z + M[4 * r + 3]);
                for (int r = 0; r < 3; r++) {
                    if (first || p[r] < o.a[r]) o.a[r] = p[r];
                    if (first || p[r] > o.g[r]) o.g[r] = p[r];
                }
                first = false;
            }
    return o;
}

}  // namespace yr

YR_API yr_status yr_instance_bound(const float *bound, const float *matrix, float *out) {
    if (!bound || !matrix || !out) return YR_ERR_INVALID_ARG;
    yr::Box b;
    std::memcpy(b.a, bound, 12);
    std::memcpy(b.g, bound + 3, 12);
    const yr::Box o = yr::instance_bound(b, matrix);
    std::memcpy(out, o.a, 12);
    std::memcpy(out + 3, o.g, 12);
    return YR_OK;
}
