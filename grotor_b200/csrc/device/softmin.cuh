// softmin.cuh -- temperature-tau soft-min version of the L-shape routing DAG
// and its hand-written adjoint.
//
// The DAG is the L-shape DP of lshape_thread.cuh:18-171 (and of lshape.cuh
// here): per tree node a table of via-stack layer ranges [lo, hi]; per tree
// edge the child's best range through each layer (cur), the arrival cost on
// each parent layer (a straight wire, or an L through one corner with its via
// stack), and the arrival over each parent range.  Every `min` of that DP is
// replaced by
//     smin(v) = m - tau * log(sum_k exp(-(v_k - m) / tau)),   m = min_k v_k,
// whose gradient is softmax(-v / tau); as tau -> 0 it becomes the hard min and
// the gradient the indicator of the chosen candidate.  Values >= kSoftAbsent
// (the hard DP's 1e22 infinity) are candidates that do not exist.
//
// Total routed cost F = sum over nets of the soft root value, with cost
// tables computed from the inputs in the working precision (fp32 or fp64):
//   wcost[c] = incr(c, 1) + unit_wire[c] * edge_len(c)
//   vcost[c] = half-split incr of the two edges a via lands between + unit_via
//   incr(c, k) = min(1e12, (of(d + k) - of(d)) * w_l),
//   of(d) = exp(0.5 * (d - capacity[c]))                        (capacity > 1e-3)
// (full_update.cuh:9-83 without the float narrowing, so FD checks in fp64 are
// smooth).  Demand d is the context's current demand, held fixed.
//
// Memory: the forward keeps only each net's root value; the backward
// recomputes each net's DP tables in a per-thread scratch slot (N * L * L
// values for the forward ranges, as many for their adjoints), so memory is
// bounded by the threads in flight, not by the nets.
#pragma once
#include "common.cuh"

namespace grb {

constexpr double kSoftAbsent = 1e21;

template <class T> __device__ __forceinline__ T s_exp(T v);
template <> __device__ __forceinline__ float s_exp<float>(float v) { return expf(v); }
template <> __device__ __forceinline__ double s_exp<double>(double v) { return exp(v); }
template <class T> __device__ __forceinline__ T s_log(T v);
template <> __device__ __forceinline__ float s_log<float>(float v) { return logf(v); }
template <> __device__ __forceinline__ double s_log<double>(double v) { return log(v); }

template <class T>
struct Soft {
    const T* cap;        // [cells]
    const T* uw;         // [cells] unit wire cost per edge
    T uv;                // unit via cost
    T tau;
    T* wc;               // [cells] wire cost
    T* vc;               // [cells] via cost
    T* P;                // [cells] exclusive prefix of wc along each track
    T* dP;               // [cells] adjoint of P
    T* dvc;              // [cells] adjoint of vc
    T* slot;             // scratch: 2 * L * L values per node (range tables, adjoints)
    T* net_cost;         // [n_nets] soft root value of each net
};

template <class T>
__device__ __forceinline__ T soft_of(const Tables& Tb, T cap, T d) {
    const T scale = static_cast<T>(Tb.of_scale);
    if (cap > static_cast<T>(0.001)) {
        const T a = static_cast<T>(0.5) * (d - cap), b = scale * static_cast<T>(0.5) * (d - cap);
        return s_exp<T>(a < b ? a : b);
    }
    if (d > 0) {
        const T a = static_cast<T>(1.5) * d, b = scale * static_cast<T>(1.5) * d;
        return s_exp<T>(a < b ? a : b);
    }
    return 0;
}
// d of / d cap.
template <class T>
__device__ __forceinline__ T soft_of_dcap(const Tables& Tb, T cap, T d) {
    if (!(cap > static_cast<T>(0.001))) return 0;
    const T scale = static_cast<T>(Tb.of_scale);
    const T a = static_cast<T>(0.5) * (d - cap), b = scale * static_cast<T>(0.5) * (d - cap);
    return a < b ? static_cast<T>(-0.5) * s_exp<T>(a) : -scale * static_cast<T>(0.5) * s_exp<T>(b);
}
template <class T>
__device__ __forceinline__ T soft_incr(const Tables& Tb, const Soft<T>& S, int c, int l, T k) {
    const T d = static_cast<T>(Tb.demand[c]) * static_cast<T>(0.5);
    const T v = (soft_of<T>(Tb, S.cap[c], d + k) - soft_of<T>(Tb, S.cap[c], d)) * static_cast<T>(Tb.short_costs[l]);
    return v < static_cast<T>(1e12) ? v : static_cast<T>(1e12);
}
template <class T>
__device__ __forceinline__ T soft_incr_dcap(const Tables& Tb, const Soft<T>& S, int c, int l, T k) {
    const T d = static_cast<T>(Tb.demand[c]) * static_cast<T>(0.5);
    const T v = (soft_of<T>(Tb, S.cap[c], d + k) - soft_of<T>(Tb, S.cap[c], d)) * static_cast<T>(Tb.short_costs[l]);
    if (!(v < static_cast<T>(1e12))) return 0;
    return (soft_of_dcap<T>(Tb, S.cap[c], d + k) - soft_of_dcap<T>(Tb, S.cap[c], d)) * static_cast<T>(Tb.short_costs[l]);
}
__device__ __forceinline__ int soft_edge_len(const Tables& Tb, int l, int x, int y) {
    if (!along_y(Tb, l)) return x < Tb.X - 1 ? Tb.xlen[x] : 0;
    return y < Tb.Y - 1 ? Tb.ylen[y] : 0;
}

// Cost tables of one cell.
template <class T>
__device__ __forceinline__ void soft_tables_cell(const Tables& Tb, const Soft<T>& S, int c) {
    const int l = c / Tb.XY, rem = c - l * Tb.XY, x = rem / Tb.Y, y = rem - x * Tb.Y;
    S.wc[c] = soft_incr<T>(Tb, S, c, l, 1) + S.uw[c] * static_cast<T>(soft_edge_len(Tb, l, x, y));
    const bool ay = along_y(Tb, l);
    const int pos = ay ? y : x, len = ay ? Tb.Y : Tb.X, stride = ay ? 1 : Tb.Y;
    T v;
    if (pos == 0) v = soft_incr<T>(Tb, S, c, l, 1);
    else if (pos == len - 1) v = soft_incr<T>(Tb, S, c - stride, l, 1);
    else v = soft_incr<T>(Tb, S, c, l, static_cast<T>(0.5)) + soft_incr<T>(Tb, S, c - stride, l, static_cast<T>(0.5));
    S.vc[c] = v + S.uv;
}

// Soft minimum of v[0..n) (entries >= kSoftAbsent do not exist); writes the
// softmax weights into w when given.  Returns kSoftAbsent * 10 when empty.
template <class T>
__device__ __forceinline__ T smin(const T* v, int n, T tau, T* w) {
    T m = static_cast<T>(kSoftAbsent);
    for (int k = 0; k < n; ++k) m = v[k] < m ? v[k] : m;
    if (!(m < static_cast<T>(kSoftAbsent))) {
        if (w) for (int k = 0; k < n; ++k) w[k] = 0;
        return static_cast<T>(kSoftAbsent) * 10;
    }
    T s = 0;
    for (int k = 0; k < n; ++k)
        if (v[k] < static_cast<T>(kSoftAbsent)) s += s_exp<T>(-(v[k] - m) / tau);
    if (w)
        for (int k = 0; k < n; ++k) w[k] = v[k] < static_cast<T>(kSoftAbsent) ? s_exp<T>(-(v[k] - m) / tau) / s : 0;
    return m - tau * s_log<T>(s);
}

template <class T>
__device__ __forceinline__ T soft_wire(const Tables& Tb, const Soft<T>& S, int l, int xmin, int xmax, int ymin, int ymax) {
    return S.P[cell_index(Tb, l, xmax, ymax)] - S.P[cell_index(Tb, l, xmin, ymin)];
}
template <class T>
__device__ __forceinline__ void soft_wire_adj(const Tables& Tb, const Soft<T>& S, int l, int xmin, int xmax, int ymin,
                                              int ymax, T g) {
    if (g == 0 || (xmin == xmax && ymin == ymax)) return;
    atomicAdd(S.dP + cell_index(Tb, l, xmax, ymax), g);
    atomicAdd(S.dP + cell_index(Tb, l, xmin, ymin), -g);
}

// Candidate set of one tree edge: the arrival on parent layer pl from child
// layer cl.  Straight edges have the single candidate cl == pl (layers of the
// edge's direction); L edges every cl of the other parity (lshape_thread.cuh).
struct SoftEdge {
    int x, y, px, py, minx, maxx, miny, maxy;
    bool straight;
};

// Candidate cost excluding cur[cl]; NaN-free, absent when not a candidate.
template <class T>
__device__ __forceinline__ T soft_leg(const Tables& Tb, const Soft<T>& S, const SoftEdge& E, int cl, int pl) {
    const int L = Tb.L;
    (void)L;
    if (E.straight) {
        if (cl != pl) return static_cast<T>(kSoftAbsent) * 10;
        if (!along_y(Tb, cl) && E.y != E.py) return static_cast<T>(kSoftAbsent) * 10;
        if (along_y(Tb, cl) && E.x != E.px) return static_cast<T>(kSoftAbsent) * 10;
        return soft_wire<T>(Tb, S, cl, E.minx, E.maxx, E.miny, E.maxy);
    }
    if (((cl ^ pl) & 1) == 0) return static_cast<T>(kSoftAbsent) * 10;
    T cost = along_y(Tb, cl) ? soft_wire<T>(Tb, S, cl, E.x, E.x, E.miny, E.maxy)
                             : soft_wire<T>(Tb, S, cl, E.minx, E.maxx, E.y, E.y);
    T cost2 = 0;
    for (int l = min(cl, pl) + 1; l < max(cl, pl); ++l)
        cost2 += along_y(Tb, cl) ? S.vc[cell_index(Tb, l, E.x, E.py)] : S.vc[cell_index(Tb, l, E.px, E.y)];
    cost2 += along_y(Tb, pl) ? soft_wire<T>(Tb, S, pl, E.px, E.px, E.miny, E.maxy)
                             : soft_wire<T>(Tb, S, pl, E.minx, E.maxx, E.py, E.py);
    return cost + cost2;
}
template <class T>
__device__ __forceinline__ void soft_leg_adj(const Tables& Tb, const Soft<T>& S, const SoftEdge& E, int cl, int pl, T g) {
    if (g == 0) return;
    if (E.straight) {
        soft_wire_adj<T>(Tb, S, cl, E.minx, E.maxx, E.miny, E.maxy, g);
        return;
    }
    if (along_y(Tb, cl)) soft_wire_adj<T>(Tb, S, cl, E.x, E.x, E.miny, E.maxy, g);
    else soft_wire_adj<T>(Tb, S, cl, E.minx, E.maxx, E.y, E.y, g);
    for (int l = min(cl, pl) + 1; l < max(cl, pl); ++l)
        atomicAdd(S.dvc + (along_y(Tb, cl) ? cell_index(Tb, l, E.x, E.py) : cell_index(Tb, l, E.px, E.y)), g);
    if (along_y(Tb, pl)) soft_wire_adj<T>(Tb, S, pl, E.px, E.px, E.miny, E.maxy, g);
    else soft_wire_adj<T>(Tb, S, pl, E.minx, E.maxx, E.py, E.py, g);
}

__device__ __forceinline__ SoftEdge soft_edge(const Tables& Tb, int node, int par) {
    SoftEdge E;
    E.x = node / Tb.Y % Tb.X; E.y = node % Tb.Y;
    E.px = par / Tb.Y % Tb.X; E.py = par % Tb.Y;
    E.minx = min(E.x, E.px); E.maxx = max(E.x, E.px); E.miny = min(E.y, E.py); E.maxy = max(E.y, E.py);
    E.straight = E.x == E.px || E.y == E.py;
    return E;
}

// Forward DP of one net into dist[N][L][L] (its final range tables); returns
// the soft root value.
template <class T>
__device__ T soft_net_forward(const Tables& Tb, const Soft<T>& S, const Plan& P, int id, T* dist) {
    const int L = Tb.L, LL = L * L;
    const int nb = P.node_off[id], N = P.node_off[id + 1] - nb;
    const T absent = static_cast<T>(kSoftAbsent) * 10;
    for (int i = 0; i < N; ++i) {
        const int v = P.nodes[nb + i], lp = v / Tb.XY, x = v / Tb.Y % Tb.X, y = v % Tb.Y;
        T* d = dist + size_t(i) * LL;
        for (int lo = 0; lo < L; ++lo) {
            d[lo * L + lo] = 0;
            for (int hi = lo + 1; hi < L; ++hi) d[lo * L + hi] = d[lo * L + hi - 1] + S.vc[cell_index(Tb, hi - 1, x, y)];
            for (int hi = 0; hi < lo; ++hi) d[lo * L + hi] = absent;
            if (lp < L)
                for (int hi = lo; hi < L; ++hi)
                    if (lo > lp || hi < lp) d[lo * L + hi] = absent;
        }
    }
    T vals[kMaxLayers * kMaxLayers];
    for (int i = N - 1; i >= 1; --i) {
        const int p = P.parents[nb + i];
        const SoftEdge E = soft_edge(Tb, P.nodes[nb + i], P.nodes[nb + p]);
        const T* di = dist + size_t(i) * LL;
        T cur[kMaxLayers], diag[kMaxLayers];
        for (int l = 0; l < L; ++l) {
            int n = 0;
            for (int lo = 0; lo <= l; ++lo)
                for (int hi = l; hi < L; ++hi) vals[n++] = di[lo * L + hi];
            cur[l] = smin<T>(vals, n, S.tau, nullptr);
        }
        for (int pl = 0; pl < L; ++pl) {
            for (int cl = 0; cl < L; ++cl) vals[cl] = cur[cl] + soft_leg<T>(Tb, S, E, cl, pl);
            diag[pl] = smin<T>(vals, L, S.tau, nullptr);
        }
        T* dp = dist + size_t(p) * LL;
        for (int lo = 0; lo < L; ++lo)
            for (int hi = lo; hi < L; ++hi) dp[lo * L + hi] += smin<T>(diag + lo, hi - lo + 1, S.tau, nullptr);
    }
    int n = 0;
    for (int lo = 0; lo < L; ++lo)
        for (int hi = lo; hi < L; ++hi) vals[n++] = dist[lo * L + hi];
    return smin<T>(vals, n, S.tau, nullptr);
}

// Adjoint of one net: recomputes the forward ranges, then propagates g (the
// gradient of F with respect to the net's root value) to the tables.
template <class T>
__device__ void soft_net_backward(const Tables& Tb, const Soft<T>& S, const Plan& P, int id, T* dist, T* gd, T g) {
    const int L = Tb.L, LL = L * L;
    const int nb = P.node_off[id], N = P.node_off[id + 1] - nb;
    soft_net_forward<T>(Tb, S, P, id, dist);
    for (size_t k = 0; k < size_t(N) * LL; ++k) gd[k] = 0;
    T vals[kMaxLayers * kMaxLayers], w[kMaxLayers * kMaxLayers];
    {
        int n = 0;
        for (int lo = 0; lo < L; ++lo)
            for (int hi = lo; hi < L; ++hi) vals[n++] = dist[lo * L + hi];
        smin<T>(vals, n, S.tau, w);
        n = 0;
        for (int lo = 0; lo < L; ++lo)
            for (int hi = lo; hi < L; ++hi) gd[lo * L + hi] = g * w[n++];
    }
    // Edges in the reverse of the forward order: a node's range adjoint is
    // complete once its own parent edge has been processed.
    for (int i = 1; i < N; ++i) {
        const int p = P.parents[nb + i];
        const SoftEdge E = soft_edge(Tb, P.nodes[nb + i], P.nodes[nb + p]);
        const T* di = dist + size_t(i) * LL;
        const T* gp = gd + size_t(p) * LL;
        T* gi = gd + size_t(i) * LL;
        T cur[kMaxLayers], diag[kMaxLayers], gdiag[kMaxLayers], gcur[kMaxLayers];
        for (int l = 0; l < L; ++l) {
            int n = 0;
            for (int lo = 0; lo <= l; ++lo)
                for (int hi = l; hi < L; ++hi) vals[n++] = di[lo * L + hi];
            cur[l] = smin<T>(vals, n, S.tau, nullptr);
            gcur[l] = 0;
            gdiag[l] = 0;
        }
        for (int pl = 0; pl < L; ++pl) {
            for (int cl = 0; cl < L; ++cl) vals[cl] = cur[cl] + soft_leg<T>(Tb, S, E, cl, pl);
            diag[pl] = smin<T>(vals, L, S.tau, nullptr);
        }
        // parent range [lo, hi] += smin(diag[lo..hi])
        for (int lo = 0; lo < L; ++lo)
            for (int hi = lo; hi < L; ++hi) {
                const T gr = gp[lo * L + hi];
                if (gr == 0) continue;
                smin<T>(diag + lo, hi - lo + 1, S.tau, w);
                for (int k = 0; k <= hi - lo; ++k) gdiag[lo + k] += gr * w[k];
            }
        // arrival on pl from child layer cl
        for (int pl = 0; pl < L; ++pl) {
            if (gdiag[pl] == 0) continue;
            T legs[kMaxLayers];
            for (int cl = 0; cl < L; ++cl) {
                legs[cl] = soft_leg<T>(Tb, S, E, cl, pl);
                vals[cl] = cur[cl] + legs[cl];
            }
            smin<T>(vals, L, S.tau, w);
            for (int cl = 0; cl < L; ++cl) {
                if (w[cl] == 0) continue;
                gcur[cl] += gdiag[pl] * w[cl];
                soft_leg_adj<T>(Tb, S, E, cl, pl, gdiag[pl] * w[cl]);
            }
        }
        // cur[l] = smin over the child's ranges containing l
        for (int l = 0; l < L; ++l) {
            if (gcur[l] == 0) continue;
            int n = 0;
            for (int lo = 0; lo <= l; ++lo)
                for (int hi = l; hi < L; ++hi) vals[n++] = di[lo * L + hi];
            smin<T>(vals, n, S.tau, w);
            n = 0;
            for (int lo = 0; lo <= l; ++lo)
                for (int hi = l; hi < L; ++hi) gi[lo * L + hi] += gcur[l] * w[n++];
        }
    }
    // Via stacks of every node's ranges.
    for (int i = 0; i < N; ++i) {
        const int v = P.nodes[nb + i], x = v / Tb.Y % Tb.X, y = v % Tb.Y;
        const T* gi = gd + size_t(i) * LL;
        const T* di = dist + size_t(i) * LL;
        for (int l = 0; l + 1 < L; ++l) {
            T acc = 0;  // every finite range [lo, hi] with lo <= l < hi holds vc[l]
            for (int lo = 0; lo <= l; ++lo)
                for (int hi = l + 1; hi < L; ++hi)
                    if (di[lo * L + hi] < static_cast<T>(kSoftAbsent)) acc += gi[lo * L + hi];
            if (acc != 0) atomicAdd(S.dvc + cell_index(Tb, l, x, y), acc);
        }
    }
}

}  // namespace grb
