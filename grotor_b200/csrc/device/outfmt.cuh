// outfmt.cuh -- the .out text of routed nets, formatted on the device.
//
// Semantics of the reference's writer (graph::output_nets, output.hpp:79-112,
// grotor::RouteWriter, output_writer.hpp:29-43): per output record its name,
// "\n(\n", then one line "x0 y0 l0 x1 y1 l1\n" per segment -- first a via
// (pin, pin + X*Y) for every pin on layer 0, then the record's extra route
// pairs, then every subnet's route words (pairs shifted up one layer, + X*Y;
// phase-two words for rerouted subnets) -- and ")\n".  Each segment is
// written with the smaller 3-D position first; a position p is
// (p / Y % X, p % Y, p / (X*Y)); numbers are decimal without leading zeros
// (std::to_chars of a non-negative int).
//
// B200 form: one warp per record in two passes -- byte count (lanes take
// segments, a warp sum) and, after an exclusive scan of the counts, the text
// (lanes take segments and write their lines at the offsets of a warp scan;
// the name is copied by all lanes).
#pragma once
#include "common.cuh"

namespace grb {

struct OutRecords {
    int n, X, Y;
    const long long* name_off;   // [n+1]
    const char* names;
    const int* pin_off;          // [n+1]
    const int* pins;
    const int* extra_off;        // [n+1], two positions per segment
    const int* extra;
    const int* sub_off;          // [n+1]
    const int* subnets;
    const unsigned char* sub_phase2;
    const long long* route_off;  // stage-one routes of the context
    const int* routes;
    const long long* route2_off; // phase-two routes (nullptr when none)
    const int* routes2;
    long long* bytes;            // [n+1] per record, scanned in place into offsets
    char* text;
    int* status;                 // [0] code (1 subnet id, 2 route words), [1] record
    int n_nets;
};

__device__ __forceinline__ int dec_len(unsigned v) {
    int d = 1;
    while (v >= 10) { v /= 10; ++d; }
    return d;
}
__device__ __forceinline__ char* dec_put(char* p, unsigned v) {
    const int d = dec_len(v);
    for (int i = d - 1; i >= 0; --i) { p[i] = static_cast<char>('0' + v % 10); v /= 10; }
    return p + d;
}

// One segment line of positions a, b (3-D, non-negative).
struct OutLine {
    unsigned v[6];
};
__device__ __forceinline__ OutLine out_line(const OutRecords& R, int a, int b) {
    if (a > b) { const int t = a; a = b; b = t; }
    const int XY = R.X * R.Y;
    OutLine L;
    L.v[0] = a / R.Y % R.X; L.v[1] = a % R.Y; L.v[2] = a / XY;
    L.v[3] = b / R.Y % R.X; L.v[4] = b % R.Y; L.v[5] = b / XY;
    return L;
}
__device__ __forceinline__ int out_line_len(const OutLine& L) {
    int n = 6;
#pragma unroll
    for (int k = 0; k < 6; ++k) n += dec_len(L.v[k]);
    return n;
}
__device__ __forceinline__ void out_line_put(char* p, const OutLine& L) {
#pragma unroll
    for (int k = 0; k < 6; ++k) {
        p = dec_put(p, L.v[k]);
        *p++ = k == 5 ? '\n' : ' ';
    }
}

// Record r's segment lines in output order, 32 at a time: every lane calls
// g(on, line) once per group, `on` when the lane holds a line of the group
// (lane order is output order inside a group).  False when a subnet id or
// its route words are invalid.
template <class G>
__device__ __forceinline__ bool out_groups(const OutRecords& R, int r, int lane, G g) {
    const int XY = R.X * R.Y;
    for (int base = R.pin_off[r]; base < R.pin_off[r + 1]; base += 32) {  // pins on layer 0: a via up
        const int q = base + lane;
        const bool on = q < R.pin_off[r + 1] && R.pins[q] >= 0 && R.pins[q] < XY;
        g(on, on ? out_line(R, R.pins[q], R.pins[q] + XY) : OutLine{});
    }
    for (int base = R.extra_off[r]; base + 1 < R.extra_off[r + 1]; base += 64) {
        const int q = base + 2 * lane;
        const bool on = q + 1 < R.extra_off[r + 1];
        g(on, on ? out_line(R, R.extra[q], R.extra[q + 1]) : OutLine{});
    }
    for (int s = R.sub_off[r]; s < R.sub_off[r + 1]; ++s) {
        const int id = R.subnets[s];
        if (id < 0 || id >= R.n_nets) return false;
        const bool two = R.sub_phase2[s] != 0;
        if (two && !R.routes2) return false;
        const int* w = two ? R.routes2 + R.route2_off[id] : R.routes + R.route_off[id];
        const long long cap = two ? R.route2_off[id + 1] - R.route2_off[id] : R.route_off[id + 1] - R.route_off[id];
        if (cap < 1 || w[0] < 1 || w[0] > cap) return false;
        const int segs = (w[0] - 1) / 2;
        for (int base = 0; base < segs; base += 32) {
            const int j = base + lane;
            const bool on = j < segs;
            g(on, on ? out_line(R, w[1 + 2 * j] + XY, w[2 + 2 * j] + XY) : OutLine{});
        }
    }
    return true;
}

// Pass 1: bytes of record r (warp).
__device__ __forceinline__ void out_count(const OutRecords& R, int r, int lane) {
    long long sum = 0;
    const bool ok = out_groups(R, r, lane, [&](bool on, const OutLine& L) { if (on) sum += out_line_len(L); });
    for (int o = 16; o; o >>= 1) sum += __shfl_xor_sync(0xffffffffu, sum, o);
    if (lane == 0) {
        if (!ok && atomicCAS(R.status, 0, 1) == 0) R.status[1] = r;
        R.bytes[r] = ok ? sum + (R.name_off[r + 1] - R.name_off[r]) + 5 : 0;
    }
}

// Pass 2: the text of record r at its scanned offset (warp; only after a
// pass 1 without errors).  Each group's lines are placed by a warp scan of
// their lengths.
__device__ __forceinline__ void out_write(const OutRecords& R, int r, int lane) {
    char* p = R.text + R.bytes[r];
    const long long nl = R.name_off[r + 1] - R.name_off[r];
    for (long long i = lane; i < nl; i += 32) p[i] = R.names[R.name_off[r] + i];
    p += nl;
    if (lane == 0) { p[0] = '\n'; p[1] = '('; p[2] = '\n'; }
    p += 3;
    long long done = 0;
    out_groups(R, r, lane, [&](bool on, const OutLine& L) {
        const int len = on ? out_line_len(L) : 0;
        int incl = len;
        for (int o = 1; o < 32; o <<= 1) {
            const int v = __shfl_up_sync(0xffffffffu, incl, o);
            if (lane >= o) incl += v;
        }
        if (on) out_line_put(p + done + incl - len, L);
        done += __shfl_sync(0xffffffffu, incl, 31);
    });
    if (lane == 0) { p[done] = ')'; p[done + 1] = '\n'; }
}

}  // namespace grb
