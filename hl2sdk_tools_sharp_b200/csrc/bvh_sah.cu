// bvh_sah.cu -- top-down surface-area-heuristic BVH over padded triangle
// boxes, on the host.  Ranges of up to kSweep triangles try every split
// position along each axis (the triangles sorted by box centre); larger
// ranges bin the centres (kBins per axis).  A range becomes a leaf when it
// holds at most kMaxLeaf triangles and testing them all is no dearer than
// the best split.  Costs: one unit per node visit, one per triangle test.
//
// The answers of a walk do not depend on the tree's shape (it tests every
// triangle whose padded box the segment meets); the shape only decides how
// many nodes and triangles a walk visits.
//
// The top three levels are split on the calling thread; the ranges below
// them are built as tasks on the host's threads, each into its own node
// list, and the lists are spliced back in the serial build's preorder, so
// the tree is the one a single thread builds (8x8 room grid, 9,144
// triangles: 13.5 ms serial, 3.8 ms on eight threads).

#include <algorithm>
#include <cfloat>
#include <climits>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <numeric>
#include <vector>

#include "bvh_sah.h"
#include "host_parallel.h"
#include "vrad_internal.cuh"

namespace vrad {

namespace {

constexpr int32_t kSweep = 2048;
constexpr int kBins = 32;
constexpr double kCostNode = 1.0, kCostTri = 1.0;

struct Box {
    float lo[3] = {FLT_MAX, FLT_MAX, FLT_MAX};
    float hi[3] = {-FLT_MAX, -FLT_MAX, -FLT_MAX};
    void grow(const Box &b) {
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], b.lo[a]);
            hi[a] = std::max(hi[a], b.hi[a]);
        }
    }
    void grow(const float p[3]) {
        for (int a = 0; a < 3; a++) {
            lo[a] = std::min(lo[a], p[a]);
            hi[a] = std::max(hi[a], p[a]);
        }
    }
    double half_area() const {
        if (lo[0] > hi[0]) return 0.0;
        const double dx = (double)hi[0] - lo[0], dy = (double)hi[1] - lo[1], dz = (double)hi[2] - lo[2];
        return dx * dy + dy * dz + dz * dx;
    }
};

int32_t ceil_log2(int32_t m) {
    int32_t k = 0;
    while ((int64_t)1 << k < m) k++;
    return k;
}

// One subtree's output: its inner nodes in preorder (child references
// local to it: inner nodes by index, leaves as leaf_ref into the shared
// order), and its statistics.
struct Sink {
    std::vector<float4> nodes;
    int32_t inner = 0, leaves = 0, max_leaf = 0, depth = 0;
    double cost = 0.0;
};

// A range left for a worker: built on its own, then spliced in.
struct Task {
    int32_t b, e, depth;
};

// Ranges at this depth, or this small, below the top of the tree are built
// as tasks, in parallel on the host's threads.
constexpr int32_t kTaskDepth = 3;
constexpr int32_t kTaskMin = 256;

class Builder {
public:
    Builder(const float *box, int32_t n, SahTree &out) : out_(out), n_(n) {
        boxes_.resize((size_t)n);
        cen_.resize((size_t)n * 3);
        for (int32_t i = 0; i < n; i++) {
            Box &b = boxes_[(size_t)i];
            for (int a = 0; a < 3; a++) {
                b.lo[a] = box[6 * (size_t)i + a];
                b.hi[a] = box[6 * (size_t)i + 3 + a];
                cen_[3 * (size_t)i + a] = 0.5f * (b.lo[a] + b.hi[a]);
            }
        }
        out_.order.resize((size_t)n);
        std::iota(out_.order.begin(), out_.order.end(), 0);
        out_.nodes.clear();
        out_.nodes.reserve((size_t)4 * (n > 1 ? n - 1 : 1));
        out_.inner = out_.leaves = out_.max_leaf = out_.depth = 0;
        out_.sah_cost = 0.0;
    }

    // The top of the tree serially down to the tasks, the tasks on the
    // host's threads (each on its own range of the order), then every node
    // written out in the serial build's preorder: the tree is the one a
    // single thread builds.
    void run(bool parallel) {
        Box root;
        top_.nodes.clear();
        // (Task references sit below every leaf reference while 8 n stays
        // well inside an int.)
        build(0, n_, 0, true, root, top_, parallel && n_ < (1 << 27) ? &tasks_ : nullptr);
        task_sink_.assign(tasks_.size(), Sink());
        task_root_.assign(tasks_.size(), 0);
        parallel_for((int64_t)tasks_.size(), 1, [&](int64_t k) {
            Box bx;
            const Task &t = tasks_[(size_t)k];
            task_root_[(size_t)k] = build(t.b, t.e, t.depth, false, bx, task_sink_[(size_t)k], nullptr);
        });
        emit_top(0);
        double cost = top_.cost;
        out_.leaves = top_.leaves;
        out_.max_leaf = top_.max_leaf;
        out_.depth = top_.depth;
        for (const Sink &sk : task_sink_) {
            cost += sk.cost;
            out_.leaves += sk.leaves;
            out_.max_leaf = std::max(out_.max_leaf, sk.max_leaf);
            out_.depth = std::max(out_.depth, sk.depth);
        }
        root_area_ = root.half_area();
        out_.sah_cost = root_area_ > 0.0 ? cost / root_area_ : 0.0;
    }

private:
    // A task's reference in the top part: below every leaf reference.
    static int32_t task_ref(size_t k) { return INT32_MIN + (int32_t)k; }

    // Builds [b, e) into sink, returns its reference (an inner node's
    // index in sink, a leaf reference, or, with tasks, a task's) and its box.
    int32_t build(int32_t b, int32_t e, int32_t depth, bool root, Box &bx, Sink &sink, std::vector<Task> *tasks) {
        const int32_t m = e - b;
        if (tasks && !root && (depth >= kTaskDepth || m <= kTaskMin)) {
            bx = Box();
            const int32_t *idx = out_.order.data();
            for (int32_t k = b; k < e; k++) bx.grow(boxes_[(size_t)idx[k]]);
            tasks->push_back(Task{b, e, depth});
            return task_ref(tasks->size() - 1);
        }
        int32_t mid = 0;
        const bool leaf = choose(b, e, depth, root, mid, bx);
        if (leaf) {
            sink.leaves++;
            sink.max_leaf = std::max(sink.max_leaf, m);
            sink.cost += kCostTri * m * bx.half_area();
            return leaf_ref(b, m);
        }
        const int32_t me = sink.inner++;
        sink.nodes.resize((size_t)4 * sink.inner);
        sink.depth = std::max(sink.depth, depth + 1);
        sink.cost += kCostNode * bx.half_area();
        Box b0, b1;
        const int32_t r0 = build(b, mid, depth + 1, false, b0, sink, tasks);
        const int32_t r1 = build(mid, e, depth + 1, false, b1, sink, tasks);
        float4 *nd = &sink.nodes[(size_t)4 * me];
        nd[0] = make_float4(b0.lo[0], b0.hi[0], b0.lo[1], b0.hi[1]);
        nd[1] = make_float4(b1.lo[0], b1.hi[0], b1.lo[1], b1.hi[1]);
        nd[2] = make_float4(b0.lo[2], b0.hi[2], b1.lo[2], b1.hi[2]);
        float f0, f1;
        std::memcpy(&f0, &r0, 4);
        std::memcpy(&f1, &r1, 4);
        nd[3] = make_float4(f0, f1, 0.0f, 0.0f);
        return me;
    }

    // Writes top node i and everything below it into out_, in preorder;
    // returns its index there.
    int32_t emit_top(int32_t i) {
        const int32_t me = out_.inner++;
        out_.nodes.resize((size_t)4 * out_.inner);
        const float4 *src = &top_.nodes[(size_t)4 * i];
        int32_t ref[2];
        std::memcpy(&ref[0], &src[3].x, 4);
        std::memcpy(&ref[1], &src[3].y, 4);
        for (int c = 0; c < 2; c++) {
            if (ref[c] >= 0) ref[c] = emit_top(ref[c]);
            else if (ref[c] < task_ref(0) + (int32_t)tasks_.size()) ref[c] = emit_task((size_t)(ref[c] - task_ref(0)));
        }
        float4 *nd = &out_.nodes[(size_t)4 * me];
        nd[0] = src[0];
        nd[1] = src[1];
        nd[2] = src[2];
        float f0, f1;
        std::memcpy(&f0, &ref[0], 4);
        std::memcpy(&f1, &ref[1], 4);
        nd[3] = make_float4(f0, f1, 0.0f, 0.0f);
        return me;
    }

    // Appends task k's nodes to out_ with their inner references moved to
    // out_'s indices; returns its root's reference.
    int32_t emit_task(size_t k) {
        const Sink &sk = task_sink_[k];
        const int32_t root = task_root_[k];
        if (root < 0) return root;  // a leaf
        const int32_t at = out_.inner;
        out_.inner += sk.inner;
        out_.nodes.resize((size_t)4 * out_.inner);
        for (int32_t j = 0; j < sk.inner; j++) {
            float4 *nd = &out_.nodes[(size_t)4 * (at + j)];
            const float4 *src = &sk.nodes[(size_t)4 * j];
            nd[0] = src[0];
            nd[1] = src[1];
            nd[2] = src[2];
            int32_t r[2];
            std::memcpy(&r[0], &src[3].x, 4);
            std::memcpy(&r[1], &src[3].y, 4);
            for (int c = 0; c < 2; c++)
                if (r[c] >= 0) r[c] += at;
            float f0, f1;
            std::memcpy(&f0, &r[0], 4);
            std::memcpy(&f1, &r[1], 4);
            nd[3] = make_float4(f0, f1, 0.0f, 0.0f);
        }
        return at + root;
    }

    // Leaf or split of [b, e); on a split, reorders the range and sets mid.
    bool choose(int32_t b, int32_t e, int32_t depth, bool root, int32_t &mid, Box &bx) {
        int32_t *idx = out_.order.data();
        const int32_t m = e - b;
        Box cb;
        bx = Box();
        for (int32_t k = b; k < e; k++) {
            bx.grow(boxes_[(size_t)idx[k]]);
            cb.grow(&cen_[3 * (size_t)idx[k]]);
        }
        if (m == 1) return true;
        const bool must_split = root || m > kMaxLeaf;
        // Depth guard: a range that could not finish within the walk's
        // stack by halving is halved from here on.
        if (depth + 1 + ceil_log2(m) >= kStackDepth) {
            if (!must_split) return true;
            median(b, e, cb, mid);
            return false;
        }
        const double area = std::max(bx.half_area(), 1e-30);
        double best = INFINITY;
        int best_axis = -1;
        int32_t best_pos = 0;
        if (m <= kSweep) {
            std::vector<int32_t> tmp((size_t)m);
            std::vector<double> right((size_t)m);
            for (int a = 0; a < 3; a++) {
                if (!(cb.hi[a] > cb.lo[a])) continue;
                std::copy(idx + b, idx + e, tmp.begin());
                sort_axis(tmp, a);
                Box r;
                for (int32_t k = m - 1; k >= 1; k--) {
                    r.grow(boxes_[(size_t)tmp[(size_t)k]]);
                    right[(size_t)k] = r.half_area();
                }
                Box l;
                for (int32_t k = 1; k < m; k++) {
                    l.grow(boxes_[(size_t)tmp[(size_t)k - 1]]);
                    const double c = kCostNode + kCostTri * (l.half_area() * k + right[(size_t)k] * (m - k)) / area;
                    if (c < best) {
                        best = c;
                        best_axis = a;
                        best_pos = k;
                    }
                }
            }
            if (best_axis >= 0 && (must_split || best < kCostTri * m)) {
                std::copy(idx + b, idx + e, tmp.begin());
                sort_axis(tmp, best_axis);
                std::copy(tmp.begin(), tmp.end(), idx + b);
                mid = b + best_pos;
                return false;
            }
        } else {
            int best_bin = 0;
            for (int a = 0; a < 3; a++) {
                if (!(cb.hi[a] > cb.lo[a])) continue;
                Box bins[kBins];
                int32_t count[kBins] = {0};
                for (int32_t k = b; k < e; k++) {
                    const int j = bin_of(idx[k], a, cb);
                    bins[j].grow(boxes_[(size_t)idx[k]]);
                    count[j]++;
                }
                double right[kBins];
                int32_t nright[kBins];
                Box r;
                int32_t nr = 0;
                for (int j = kBins - 1; j >= 1; j--) {
                    r.grow(bins[j]);
                    nr += count[j];
                    right[j] = r.half_area();
                    nright[j] = nr;
                }
                Box l;
                int32_t nl = 0;
                for (int j = 1; j < kBins; j++) {
                    l.grow(bins[j - 1]);
                    nl += count[j - 1];
                    if (nl == 0 || nright[j] == 0) continue;
                    const double c = kCostNode + kCostTri * (l.half_area() * nl + right[j] * nright[j]) / area;
                    if (c < best) {
                        best = c;
                        best_axis = a;
                        best_bin = j;
                    }
                }
            }
            if (best_axis >= 0) {
                int32_t *p = std::partition(idx + b, idx + e,
                                            [&](int32_t t) { return bin_of(t, best_axis, cb) < best_bin; });
                mid = (int32_t)(p - idx);
                if (mid > b && mid < e) return false;
            }
        }
        if (!must_split) return true;
        median(b, e, cb, mid);
        return false;
    }

    int bin_of(int32_t t, int a, const Box &cb) const {
        const double ext = (double)cb.hi[a] - cb.lo[a];
        int j = (int)(((double)cen_[3 * (size_t)t + a] - cb.lo[a]) * kBins / ext);
        return j < 0 ? 0 : (j >= kBins ? kBins - 1 : j);
    }

    void sort_axis(std::vector<int32_t> &v, int a) const {
        std::sort(v.begin(), v.end(), [&](int32_t x, int32_t y) {
            const float cx = cen_[3 * (size_t)x + a], cy = cen_[3 * (size_t)y + a];
            return cx < cy || (cx == cy && x < y);
        });
    }

    // Halves [b, e) at the median centre of its widest centre axis (by
    // index when every centre coincides).
    void median(int32_t b, int32_t e, const Box &cb, int32_t &mid) {
        int32_t *idx = out_.order.data();
        int axis = 0;
        for (int a = 1; a < 3; a++)
            if ((double)cb.hi[a] - cb.lo[a] > (double)cb.hi[axis] - cb.lo[axis]) axis = a;
        mid = b + (e - b) / 2;
        std::nth_element(idx + b, idx + mid, idx + e, [&](int32_t x, int32_t y) {
            const float cx = cen_[3 * (size_t)x + axis], cy = cen_[3 * (size_t)y + axis];
            return cx < cy || (cx == cy && x < y);
        });
    }

    SahTree &out_;
    int32_t n_;
    std::vector<Box> boxes_;
    std::vector<float> cen_;
    double root_area_ = 0.0;
    Sink top_;
    std::vector<Task> tasks_;
    std::vector<Sink> task_sink_;
    std::vector<int32_t> task_root_;
};

}  // namespace

void build_sah(const float *box, int32_t n, SahTree &out, bool parallel) {
    Builder bld(box, n, out);
    bld.run(parallel);
}

}  // namespace vrad
