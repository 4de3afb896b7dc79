// fk_kernels.cu -- sm_100a kernels of the FK forward / adjoint engine.
//
// Every time step is one fused launch.  A CTA owns a TX x TY tile of the grid,
// stages the tile plus a HALO-wide ring of each field into shared memory once,
// and runs all four RK stages out of shared memory: stage s is evaluated on the
// tile grown by (4 - s) cells, so the halo shrinks by one cell per stage and no
// stage needs another CTA's data (temporal blocking over the RK stages).
// Global traffic per cell and step is therefore one read and one write of the
// state plus gh (56 B), instead of the reference's four launches and ~440 B
// (cu-F:766-793).
//
// The work is FP64 arithmetic (three exp-based smoothed steps and one division
// per vector-field evaluation), so the kernels are written for issue
// efficiency: stage inputs ping-pong between two shared buffers (no per-thread
// register arrays across barriers, loops stay rolled and the code fits the
// instruction cache), the step-start state is re-read from L1/L2 instead of
// occupying shared memory, and the interior accumulator is the only other
// shared buffer.
#include "fk_kernels.h"
#include "fk_bulk.cuh"

#include <cstdio>
#include <cstdlib>
#include <utility>
#include <vector>

namespace fkadj {

namespace {

// Programmatic dependent launch.  The step kernels are launched with
// programmatic stream serialisation: the next kernel in the stream may be
// launched while this one still runs.  Each step kernel first waits for the
// kernel before it to complete (its writes visible), then lets the next one be
// launched.  Execution stays in stream order; only the launch latency between
// consecutive steps overlaps the tail of the previous kernel.
__device__ __forceinline__ void pdl_enter() {
    asm volatile("griddepcontrol.wait;" ::: "memory");
    asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
}

// Cells a thread keeps in flight per stage loop iteration (independent FP64
// chains the scheduler can interleave).
#ifndef FKADJ_STAGE_UNROLL
#define FKADJ_STAGE_UNROLL 1
#endif
// Resident CTAs per SM the batched kernels' register allocation targets: the
// single-instance kernels' choice (default; the 256-thread presets then spill a
// little but keep two or three CTAs per SM, which measured faster: 32 x 128^2
// batched 0.58 s against 0.71 s, 16 x 256^2 0.48 s against 0.72 s), or 1 (no
// spills).
#ifndef FKADJ_LOAD_UNROLL
#define FKADJ_LOAD_UNROLL 4
#endif
constexpr int kLoadUnroll = FKADJ_LOAD_UNROLL;
#ifndef FKADJ_BATCH_ONE_CTA
#define FKADJ_BATCH_ONE_CTA 0
#endif
// The single-instance midpoint, adjoint-step and exact-step kernels load the
// next cell's global operands while the current one computes (adj_mid_tile's
// first loop, adj_stage, exact_stage; the batched kernels, short of registers,
// keep the plain loops).
// Measured: the same time at 512^2, where the operands stay in L2; 4 % off
// the gradient at 2048^2 (midpoint 230 -> 204 us, step 344 -> 334 us).
#ifndef FKADJ_ADJ_PREFETCH
#define FKADJ_ADJ_PREFETCH 1
#endif
// The same for the single-instance forward step (gh and the step-start
// state): measured slower (17.3 against 16.3 us at 512^2, 260 against 243 us at
// 2048^2; 101 registers against 90), so off.
#ifndef FKADJ_FWD_PREFETCH
#define FKADJ_FWD_PREFETCH 0
#endif
#define FKADJ_BATCH_MINB(tx, ty, nt) (FKADJ_BATCH_ONE_CTA ? 1 : min_blocks(tx, ty, nt))

constexpr int kStageUnroll = FKADJ_STAGE_UNROLL;

// Row and column of cell q = threadIdx.x + k NT of a region W cells wide
// (origin r0, c0), advanced by NT cells per step without a division: the
// per-cell q / W and q % W cost the forward step 5 % of its time.
template <int W, int NT>
struct RowCol {
    int r, c;
    const int c_end;
    __device__ __forceinline__ RowCol(int r0, int c0)
        : r(r0 + (int)threadIdx.x / W), c(c0 + (int)threadIdx.x % W), c_end(c0 + W) {}
    __device__ __forceinline__ void next() {
        r += NT / W;
        c += NT % W;
        if (c >= c_end) c -= W, ++r;
    }
};

// Resident CTAs per SM the register allocation targets: what shared memory
// allows for the tile (187 KB at 64x32: one CTA of 512 or 768 threads; 101 KB
// at 32x32: two; 58 KB at 32x16 and below: three).
constexpr int min_blocks(int tx, int ty, int nt) { return nt >= 512 ? 1 : (tx * ty <= 512 ? 3 : 2); }

// Copies a rows x WIDTH window of the three planes at src (row pitch ld, plane
// pitch plane) into shared memory (row pitch WIDTH, plane pitch RCAP*WIDTH,
// RCAP >= rows), with 16-byte vector loads when the window is 16-byte aligned.
template <int RCAP, int WIDTH, int NT>
__device__ __forceinline__ void load_region(double* __restrict__ dst, const double* __restrict__ src,
                                            int ld, long long plane, bool vec_ok, int rows) {
    constexpr int RN = RCAP * WIDTH;
    if (vec_ok && (WIDTH % 2) == 0) {
        constexpr int HW = WIDTH / 2;
        const int per = rows * HW;
#pragma unroll kLoadUnroll
        for (int q = threadIdx.x; q < 3 * per; q += NT) {
            const int f = q >= per ? (q >= 2 * per ? 2 : 1) : 0;
            const int rem = q - f * per;
            const int r = rem / HW, c2 = rem - r * HW;
            const double2 v = __ldg(reinterpret_cast<const double2*>(src + f * plane + (long long)r * ld) + c2);
            reinterpret_cast<double2*>(dst + f * RN + r * WIDTH)[c2] = v;
        }
    } else {
        const int per = rows * WIDTH;
#pragma unroll kLoadUnroll
        for (int q = threadIdx.x; q < 3 * per; q += NT) {
            const int f = q >= per ? (q >= 2 * per ? 2 : 1) : 0;
            const int rem = q - f * per;
            const int r = rem / WIDTH, c = rem - r * WIDTH;
            dst[f * RN + r * WIDTH + c] = __ldg(src + f * plane + (long long)r * ld + c);
        }
    }
}

// Tile loads through the bulk-copy engine (fk_bulk.cuh) in the one-tile-per-CTA
// step kernels; FKADJ_BULK_LOAD=0 keeps the vector loads everywhere.
#ifndef FKADJ_BULK_LOAD
#define FKADJ_BULK_LOAD 1
#endif

// Copies one window (d1 null) or two windows of the same shape into shared
// memory: through the bulk-copy engine when BULK and the windows start on an
// even column, else with vector loads.  Ends with the CTA synchronised.
// Returns false when the bounded wait for the bulk copies expired in any
// thread of the CTA (bulk_wait_cta): the tile is then incomplete, *fault (the
// problem's own fault word, read and cleared by the host after each call) is
// set, and the caller returns without computing or storing anything.
// A third window (d2, s2) may follow the first two.  A CTA that loads several
// tiles in turn (the batched kernels) passes `phase`, its count of bulk
// transfers so far, the same in every thread: the barrier is initialised at
// the first transfer only and each later one waits on the next phase's
// parity (a barrier is not re-initialised while in use).  After an expired
// wait *phase becomes ~0: the barrier's phase is then unknown, and the CTA's
// later tiles load with vector loads (their problems' results stay valid).
template <int RCAP, int WIDTH, int NT, bool BULK>
__device__ __forceinline__ bool load_windows(double* __restrict__ d0, const double* __restrict__ s0,
                                             double* __restrict__ d1, const double* __restrict__ s1, int ld,
                                             long long plane, bool vec_ok, int rows, unsigned* fault,
                                             double* __restrict__ d2 = nullptr,
                                             const double* __restrict__ s2 = nullptr, uint32_t* phase = nullptr) {
    // every row start 16-byte aligned, checked on the addresses themselves
    const bool aligned = vec_ok && ((reinterpret_cast<uintptr_t>(s0) | reinterpret_cast<uintptr_t>(s1) |
                                     reinterpret_cast<uintptr_t>(s2) | (uintptr_t)ld * 8u | (uintptr_t)plane * 8u) &
                                    15) == 0;
    if (BULK && FKADJ_BULK_LOAD && aligned && !(phase && *phase == ~0u)) {
        __shared__ uint64_t bar;
        const uint32_t k = phase ? *phase : 0u;
        uint32_t b;
        if (k == 0) {
            b = bulk_begin(&bar);
        } else {
            b = (uint32_t)__cvta_generic_to_shared(&bar);
            // the CTA's earlier reads and writes of these buffers (previous
            // tile) before the copies' writes through the async proxy
            asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        }
        __syncthreads();
        bulk_arrive(b, bulk_bytes<WIDTH>(rows) * (1u + (d1 ? 1u : 0u) + (d2 ? 1u : 0u)));
        __syncthreads();
        bulk_issue<RCAP, WIDTH, NT>(b, d0, s0, ld, plane, rows);
        if (d1) bulk_issue<RCAP, WIDTH, NT>(b, d1, s1, ld, plane, rows);
        if (d2) bulk_issue<RCAP, WIDTH, NT>(b, d2, s2, ld, plane, rows);
        if (phase) ++*phase;
        if (!bulk_wait_cta(b, fault, 1000000000ull, k & 1u)) {
            if (phase) *phase = ~0u;
            return false;
        }
    } else {
        load_region<RCAP, WIDTH, NT>(d0, s0, ld, plane, vec_ok, rows);
        if (d1) load_region<RCAP, WIDTH, NT>(d1, s1, ld, plane, vec_ok, rows);
        if (d2) load_region<RCAP, WIDTH, NT>(d2, s2, ld, plane, vec_ok, rows);
    }
    __syncthreads();
    return true;
}

// Fixed-order block sum (warp shuffles, then warps in order); result valid in
// thread 0.  All threads of the block must call it.
template <int NT>
__device__ __forceinline__ double block_sum(double v, double* red) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    __syncthreads();
    if (lane == 0) red[wid] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0) {
#pragma unroll
        for (int w = 0; w < NT / 32; ++w) s += red[w];
    }
    return s;
}

// Sums of a per-cell term over the 16x16 sub-blocks of a tile, in an order
// fixed by the sub-block alone (lane l adds the 8 cells of half-row l in
// column order, then a shuffle tree): the result does not depend on the tile
// preset or the thread count, so gradients are bit-identical whichever tile
// the autotuner picks.  term(r, c) takes interior coordinates and returns 0
// for cells that contribute nothing.  One partial per sub-block goes to
// row[sub-block index on the grid's 16x16 lattice].
template <int TX, int TY, int NT, class Term>
__device__ __forceinline__ void subblock_sums(Term term, double* __restrict__ row, int i0, int j0, int nsbx) {
    constexpr int SBX = TX / 16, SBY = TY / 16, NSB = SBX * SBY, NW = NT / 32;
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
    for (int b = w; b < NSB; b += NW) {
        const int by = b / SBX, bx = b - by * SBX;
        const int r = by * 16 + (lane >> 1), c0 = bx * 16 + (lane & 1) * 8;
        double s = 0.0;
#pragma unroll
        for (int k = 0; k < 8; ++k) s += term(r, c0 + k);
#pragma unroll
        for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
        if (lane == 0) row[(long long)(i0 / 16 + by) * nsbx + (j0 / 16 + bx)] = s;
    }
}

// The same on the lattice of 16-cell row segments (one partial per grid row
// and 16 columns), for tiles of any height: half-warp h takes segment b of the
// tile (rows x TX/16 segments, row-major), lane l of the half adds cell l, and
// an xor butterfly over the 16 lanes leaves the sum in lane 0 in an order fixed
// by the segment alone.  Every thread runs every round (the shuffles take the
// whole warp).  One partial per segment goes to row[(i0 + r) * nsbx + j0/16 + sx].
template <int TX, int NT, class Term>
__device__ __forceinline__ void segment_sums(Term term, double* __restrict__ row, int i0, int j0, int nsbx,
                                             int rows) {
    constexpr int SX = TX / 16, NH = NT / 16;
    const int l = threadIdx.x & 15, h = threadIdx.x >> 4;
    const int nseg = SX * rows;
    for (int b0 = 0; b0 < nseg; b0 += NH) {
        const int b = b0 + h;
        const bool on = b < nseg;
        const int r = on ? b / SX : 0, sx = on ? b - r * SX : 0;
        double s = on ? term(r, sx * 16 + l) : 0.0;
#pragma unroll
        for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
        if (on && l == 0) row[(long long)(i0 + r) * nsbx + (j0 / 16 + sx)] = s;
    }
}

// ---------------------------------------------------------------- forward

// One forward RK stage on the tile grown by E cells: k = f(src), then
//   MODE 0: dst = y0 + cY*k, D  = cD*k        (first stage)
//   MODE 1: dst = y0 + cY*k, D += cD*k        (middle stages)
//   MODE 2: out = (y0 + D) + cD*k             (last stage, interior only)
// y0 (the step-start state) comes from global memory; stage algebra and E
// sources of cu-F:459-562 / cu-F:766-793.
template <int E, int TX, int TY, int NT, int MODE, bool PF = false>
__device__ __forceinline__ void fwd_stage(const DevModel& P, const double* __restrict__ src,
                                          double* __restrict__ dst, double* __restrict__ D,
                                          const double* __restrict__ y0g, const double* __restrict__ ghs,
                                          int ld, long long plane, double Ev, double cY, double cD,
                                          double* __restrict__ out, double* __restrict__ stage_out, int rows,
                                          double* __restrict__ k_out, const uint8_t* __restrict__ fcs) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
    constexpr int W = TX + 2 * E;
    constexpr int IN = TX * TY;
    const int N = W * (rows + 2 * E);
    // the stage update of cell (r, c) from its step-start value and k
    auto finish = [&](int r, int c, int s, long long o, double a, double b, double e, double ku, double kv,
                      double kw) {
        const bool inner = (E == 0) || (r >= HALO && r < HALO + rows && c >= HALO && c < HALO + TX);
        const int d = (r - HALO) * TX + (c - HALO);
        if (MODE == 2) {
            out[o] = (a + D[d]) + cD * ku;
            out[plane + o] = (b + D[IN + d]) + cD * kv;
            out[2 * plane + o] = (e + D[2 * IN + d]) + cD * kw;
        } else {
            const double nu = a + cY * ku, nv = b + cY * kv, nw = e + cY * kw;
            dst[s] = nu;
            dst[RN + s] = nv;
            dst[2 * RN + s] = nw;
            if (inner) {
                if (MODE == 0) {
                    D[d] = cD * ku;
                    D[IN + d] = cD * kv;
                    D[2 * IN + d] = cD * kw;
                } else {
                    D[d] = D[d] + cD * ku;
                    D[IN + d] = D[IN + d] + cD * kv;
                    D[2 * IN + d] = D[2 * IN + d] + cD * kw;
                }
                if (stage_out) {  // stage state kept for the discrete adjoint
                    stage_out[o] = nu;
                    stage_out[plane + o] = nv;
                    stage_out[2 * plane + o] = nw;
                }
                if (MODE == 0 && k_out) {  // k1 = f(y, E0), kept for the adjoint midpoint
                    k_out[o] = ku;
                    k_out[plane + o] = kv;
                    k_out[2 * plane + o] = kw;
                }
            }
        }
    };
    RowCol<W, NT> rc(HALO - E, HALO - E);
    if constexpr (PF) {
        // Software-pipelined: the next cell's gh and step-start state are
        // loaded while this cell computes.
        struct Ops {
            double gv, a, b, e;
            int code;
        };
        auto fetch = [&](int r, int c, Ops& x) {
            const long long o = (long long)r * ld + c;
            x.gv = __ldg(ghs + o);
            if (MODE != 0) x.a = __ldg(y0g + o), x.b = __ldg(y0g + plane + o), x.e = __ldg(y0g + 2 * plane + o);
            x.code = fcs ? (int)__ldg(fcs + o) : -1;
        };
        Ops cur;
        if ((int)threadIdx.x < N) fetch(rc.r, rc.c, cur);
        for (int q = threadIdx.x; q < N; q += NT) {
            const int r = rc.r, c = rc.c;
            rc.next();
            Ops nxt;
            if (q + NT < N) fetch(rc.r, rc.c, nxt);
            const int s = r * RW + c;
            const long long o = (long long)r * ld + c;
            double a = cur.a, b = cur.b, e = cur.e;
            if (MODE == 0) a = src[s], b = src[RN + s], e = src[2 * RN + s];
            double ku, kv, kw;
            rhs_at<RW, RN>(P, src, s, Ev * cur.gv, ku, kv, kw, cur.code);
            finish(r, c, s, o, a, b, e, ku, kv, kw);
            cur = nxt;
        }
    } else {
#pragma unroll kStageUnroll
        for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
            const int r = rc.r, c = rc.c;
            const int s = r * RW + c;
            const long long o = (long long)r * ld + c;
            // global operands first: their latency overlaps the stencil arithmetic; the
            // first stage's source region is the step-start state itself
            const double gv = __ldg(ghs + o);
            double a, b, e;
            if (MODE == 0) {
                a = src[s], b = src[RN + s], e = src[2 * RN + s];
            } else {
                a = __ldg(y0g + o), b = __ldg(y0g + plane + o), e = __ldg(y0g + 2 * plane + o);
            }
            double ku, kv, kw;
            rhs_at<RW, RN>(P, src, s, Ev * gv, ku, kv, kw, fcs ? (int)__ldg(fcs + o) : -1);
            finish(r, c, s, o, a, b, e, ku, kv, kw);
        }
    }
    if (MODE != 2) __syncthreads();
}

// One RK4 step y -> y_out on tile (tbx, tby) of ty rows (ty <= TY; the tile
// in the last row of tiles is cut at the grid's edge).  When `stages` is
// non-null the stage states Y2 = y + dt/2 k1, Y3 = y + dt/2 k2, Y4 = y + dt k3
// are stored there too (three consecutive states), for the discrete-exact
// adjoint; when `k1` is non-null, k1 = f(y, E0) is stored there (a state).  The tile functions may run several times per CTA (batched
// kernels): they start by overwriting all the shared memory they read.
template <int TX, int TY, int NT, bool BULK = false, bool PF = false>
__device__ __forceinline__ void fwd_step_tile(const DevModel& P, const DevGrid& g, const double* __restrict__ yin,
                                              double* __restrict__ yout, const double* __restrict__ gh, double E0,
                                              double Eh, double E1, double* __restrict__ stages, int tbx, int tby,
                                              int ty, double* __restrict__ k1 = nullptr,
                                              unsigned* fault = nullptr, uint32_t* phase = nullptr) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
    extern __shared__ double4 smem_raw[];
    double* A = reinterpret_cast<double*>(smem_raw);
    double* B = A + 3 * RN;
    double* D = B + 3 * RN;
    const int i0 = tby * ty, j0 = tbx * TX;
    const int rows = min(ty, g.nrows - i0);
    // region origin: logical (i0 - HALO, j0 - HALO) = padded (i0, j0)
    const long long off = (long long)i0 * g.ld + j0;
    const bool vec_ok = ((g.ld | j0) & 1) == 0;
    if (!load_windows<RH, RW, NT, BULK>(A, yin + off, nullptr, nullptr, g.ld, g.plane, vec_ok, rows + 2 * HALO,
                                        fault, nullptr, nullptr, phase))
        return;
    const double* y0g = yin + off;
    const double* ghs = gh + off;
    const double dt = P.dt;
    const long long sst = 3 * g.plane;
    double* s2 = stages ? stages + off : nullptr;
    double* s3 = stages ? stages + sst + off : nullptr;
    double* s4 = stages ? stages + 2 * sst + off : nullptr;
    const uint8_t* fcs = g.fcode ? g.fcode + off : nullptr;
    fwd_stage<3, TX, TY, NT, 0, PF>(P, A, B, D, y0g, ghs, g.ld, g.plane, E0, dt * 0.5, 1.0 / 6.0 * dt, nullptr, s2,
                                rows, k1 ? k1 + off : nullptr, fcs);
    fwd_stage<2, TX, TY, NT, 1, PF>(P, B, A, D, y0g, ghs, g.ld, g.plane, Eh, dt * 0.5, 1.0 / 3.0 * dt, nullptr, s3,
                                rows, nullptr, fcs);
    fwd_stage<1, TX, TY, NT, 1, PF>(P, A, B, D, y0g, ghs, g.ld, g.plane, Eh, dt * 1.0, 1.0 / 3.0 * dt, nullptr, s4,
                                rows, nullptr, fcs);
    fwd_stage<0, TX, TY, NT, 2, PF>(P, B, A, D, y0g, ghs, g.ld, g.plane, E1, 0.0, dt * 1.0 / 6.0, yout + off, nullptr,
                                rows, nullptr, fcs);
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, min_blocks(TX, TY, NT))
    k_fwd_step(DevModel P, DevGrid g, const double* __restrict__ yin, double* __restrict__ yout,
               const double* __restrict__ gh, EStep E, double* __restrict__ stages, int ty,
               double* __restrict__ k1, unsigned* fault) {
    pdl_enter();
    exp_table_init();
    fwd_step_tile<TX, TY, NT, true, FKADJ_FWD_PREFETCH != 0>(P, g, yin, yout, gh, E.a(), E.b(), E.c(), stages,
                                                             blockIdx.x, blockIdx.y, ty, k1, fault);
}

// ------------------------------------------------- reference-mode adjoint

// Cached Jacobians: the seven entries of J_F(y)^T of every cell, seven planes.
__device__ __forceinline__ JacT load_jac(const double* __restrict__ Jb, long long plane, long long o) {
    JacT J;
    J.a0 = __ldg(Jb + o);
    J.a1 = __ldg(Jb + plane + o);
    J.a2 = __ldg(Jb + 2 * plane + o);
    J.a3 = __ldg(Jb + 3 * plane + o);
    J.a4 = __ldg(Jb + 4 * plane + o);
    J.a5 = __ldg(Jb + 5 * plane + o);
    J.a6 = __ldg(Jb + 6 * plane + o);
    return J;
}
__device__ __forceinline__ void store_jac(double* __restrict__ Jb, long long plane, long long o, const JacT& J) {
    Jb[o] = J.a0;
    Jb[plane + o] = J.a1;
    Jb[2 * plane + o] = J.a2;
    Jb[3 * plane + o] = J.a3;
    Jb[4 * plane + o] = J.a4;
    Jb[5 * plane + o] = J.a5;
    Jb[6 * plane + o] = J.a6;
}

// Midpoint state of step [t_{i-1}, t_i] (cu-G:1244-1301): y3 = cubic Hermite
// at 1/3 from (ya, yb, dt*f(ya), dt*f(yb)); yh = partial quartic at 1/2 plus
// (27/64) dt f(y3, E(t_{i-1}+dt/3)).  Halo 2: f(ya), f(yb) on the tile grown by
// one cell, f(y3) on the tile.
// Work shared between consecutive backward steps (same values, computed once):
//   f(yb, Eb) of step i is f(ya, Ea) of step i+1: when fin is non-null it is
//   read from there instead of evaluated, and f(ya, Ea) goes to fout;
//   f(ya, Ea) is k1 of the forward step from ya: when fa is non-null (the
//   forward recompute kept it) it is read from there too;
//   J_F(yh)^T, used by stages 2 and 3 of the adjoint step, goes to jh; yh
//   itself is stored only where yh is non-null (a step that reads the J(yh)
//   cache never reads yh).
template <int TX, int TY, int NT, bool BULK = false, bool PF = false>
__device__ __forceinline__ void adj_mid_tile(const DevModel& P, const DevGrid& g, const double* __restrict__ ya,
                                             const double* __restrict__ yb, const double* __restrict__ gh,
                                             double* __restrict__ yh, double Ea, double Eb, double E3,
                                             const HermiteW& hw, const double* __restrict__ fin,
                                             double* __restrict__ fout, double* __restrict__ jh, int tbx, int tby,
                                             int ty, const double* __restrict__ fa = nullptr,
                                             unsigned* fault = nullptr, uint32_t* phase = nullptr) {
    constexpr int H2 = 2;
    constexpr int RW = TX + 2 * H2, RH = TY + 2 * H2, RN = RW * RH;
    extern __shared__ double4 smem_raw[];
    double* A = reinterpret_cast<double*>(smem_raw);
    double* B = A + 3 * RN;
    double* C = B + 3 * RN;
    double* Q = C + 3 * RN;  // quartic part of yh on the tile, kept between the two loops
    const int i0 = tby * ty, j0 = tbx * TX;
    const int rows = min(ty, g.nrows - i0);
    // region origin: logical (i0 - 2, j0 - 2) = padded (i0 + 2, j0 + 2)
    const long long off = (long long)(i0 + HALO - H2) * g.ld + (j0 + HALO - H2);
    const bool vec_ok = ((g.ld | (j0 + HALO - H2)) & 1) == 0;
    if (!load_windows<RH, RW, NT, BULK>(A, ya + off, B, yb + off, g.ld, g.plane, vec_ok, rows + 2 * H2, fault,
                                        nullptr, nullptr, phase))
        return;
    const double dt = P.dt;
    {
        constexpr int W = TX + 2;
        const int N = W * (rows + 2);
        // Hermite parts of cell (r, c) from f(ya) = a0 and f(yb) = a1
        auto hermite = [&](int r, int c, int s, long long o, const double* a0, const double* a1) {
            const bool inner = r >= H2 && r < H2 + rows && c >= H2 && c < H2 + TX;
            if (inner && fout) {
                fout[o] = a0[0];
                fout[g.plane + o] = a0[1];
                fout[2 * g.plane + o] = a0[2];
            }
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                const double m0 = a0[f] * dt, m1 = a1[f] * dt;
                const double x0 = A[f * RN + s], x1 = B[f * RN + s];
                C[f * RN + s] = ((hw.c3[0] * x0 + hw.c3[1] * m0) + hw.c3[2] * x1) + hw.c3[3] * m1;
                if (inner) {
                    Q[f * TX * TY + (r - H2) * TX + (c - H2)] =
                        ((hw.c4[0] * x0 + hw.c4[1] * m0) + hw.c4[2] * x1) + hw.c4[3] * m1;
                }
            }
        };
        RowCol<W, NT> rc(1, 1);
        if constexpr (PF) {
            // Software-pipelined (the single-instance kernel): gh and the kept
            // f values of the next cell are loaded while this cell computes.
            struct Ops {
                double gg, a0[3], a1[3];
            };
            auto fetch = [&](int r, int c, Ops& x) {
                const long long o = off + (long long)r * g.ld + c;
                if (!fa || !fin) x.gg = __ldg(gh + o);  // only an evaluated f needs E gh
                if (fa) x.a0[0] = __ldg(fa + o), x.a0[1] = __ldg(fa + g.plane + o), x.a0[2] = __ldg(fa + 2 * g.plane + o);
                if (fin)
                    x.a1[0] = __ldg(fin + o), x.a1[1] = __ldg(fin + g.plane + o), x.a1[2] = __ldg(fin + 2 * g.plane + o);
            };
            Ops cur;
            if ((int)threadIdx.x < N) fetch(rc.r, rc.c, cur);
            for (int q = threadIdx.x; q < N; q += NT) {
                const int r = rc.r, c = rc.c;
                rc.next();
                Ops nxt;
                if (q + NT < N) fetch(rc.r, rc.c, nxt);
                const int s = r * RW + c;
                const long long o = off + (long long)r * g.ld + c;
                const int code = g.fcode ? (int)__ldg(g.fcode + o) : -1;
                if (!fa) rhs_at<RW, RN>(P, A, s, Ea * cur.gg, cur.a0[0], cur.a0[1], cur.a0[2], code);
                if (!fin) rhs_at<RW, RN>(P, B, s, Eb * cur.gg, cur.a1[0], cur.a1[1], cur.a1[2], code);
                hermite(r, c, s, o, cur.a0, cur.a1);
                cur = nxt;
            }
        } else {
#pragma unroll kStageUnroll
            for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
                const int r = rc.r, c = rc.c;
                const int s = r * RW + c;
                const long long o = off + (long long)r * g.ld + c;
                const double gg = __ldg(gh + o);
                double a0[3], a1[3];
                if (fa) {
                    a0[0] = __ldg(fa + o);
                    a0[1] = __ldg(fa + g.plane + o);
                    a0[2] = __ldg(fa + 2 * g.plane + o);
                } else {
                    rhs_at<RW, RN>(P, A, s, Ea * gg, a0[0], a0[1], a0[2], g.fcode ? (int)__ldg(g.fcode + o) : -1);
                }
                if (fin) {
                    a1[0] = __ldg(fin + o);
                    a1[1] = __ldg(fin + g.plane + o);
                    a1[2] = __ldg(fin + 2 * g.plane + o);
                } else {
                    rhs_at<RW, RN>(P, B, s, Eb * gg, a1[0], a1[1], a1[2], g.fcode ? (int)__ldg(g.fcode + o) : -1);
                }
                hermite(r, c, s, o, a0, a1);
            }
        }
    }
    __syncthreads();
    // C on the outer ring stays unset: stencils of tile cells reach one cell out.
    {
        const int N = TX * rows;
        RowCol<TX, NT> rc(H2, H2);
#pragma unroll kStageUnroll
        for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
            const int r = rc.r, c = rc.c;
            const int s = r * RW + c;
            const long long o = off + (long long)r * g.ld + c;
            double m2[3], yv[3];
            rhs_at<RW, RN>(P, C, s, E3 * __ldg(gh + o), m2[0], m2[1], m2[2], g.fcode ? (int)__ldg(g.fcode + o) : -1);
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                yv[f] = Q[f * TX * TY + (r - H2) * TX + (c - H2)] + hw.c2 * (m2[f] * dt);
                if (yh) yh[o + f * g.plane] = yv[f];
            }
            if (jh && !isnan(yv[0])) store_jac(jh, g.plane, o, fk_jacT(P, yv[0], yv[1], yv[2]));
        }
    }
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, min_blocks(TX, TY, NT))
    k_adj_mid(DevModel P, DevGrid g, const double* __restrict__ ya, const double* __restrict__ yb,
              const double* __restrict__ gh, double* __restrict__ yh, EStep E, HermiteW hw,
              const double* __restrict__ fin, double* __restrict__ fout, double* __restrict__ jh, int ty,
              const double* __restrict__ fa, unsigned* fault) {
    pdl_enter();
    exp_table_init();
    adj_mid_tile<TX, TY, NT, true, FKADJ_ADJ_PREFETCH != 0>(P, g, ya, yb, gh, yh, E.a(), E.b(), E.c(), hw, fin, fout,
                                                            jh, blockIdx.x, blockIdx.y, ty, fa, fault);
}

// One adjoint stage on the tile grown by E cells: k = L^T src + J_F(y)^T src,
// then (reference mode)
//   MODE 0: dst = z0 + cZ*k, D  = cD*k
//   MODE 1: dst = z0 + cZ*k, D += cD*k
//   MODE 2: out = (z0 + D) + cD*k; D_u <- out_u * gh (0 where NaN), the cell's
//           term of z.gh, which subblock_sums reduces afterwards
// (cu-G:1349-1427 in the order of cu-G:1885-1891).
// The Jacobian comes from the cache jload when it is non-null, else it is
// evaluated at ys; jstore (non-null only in the last stage) keeps the evaluated
// one for the next backward step.
template <int E, int TX, int TY, int NT, int MODE, bool PF = false>
__device__ __forceinline__ void adj_stage(const DevModel& P, const DevGrid& g, const double* __restrict__ src,
                                          double* __restrict__ dst, double* __restrict__ D,
                                          const double* __restrict__ z0g, const uint8_t* __restrict__ wc,
                                          const double* __restrict__ ys, long long off, double cZ, double cD,
                                          double* __restrict__ out, const double* __restrict__ gh,
                                          const double* __restrict__ jload, double* __restrict__ jstore,
                                          int rows = TY) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
    constexpr int W = TX + 2 * E;
    constexpr int IN = TX * TY;
    const int N = W * (rows + 2 * E);
    // the stage update of cell (r, c) from its step-start value and k
    auto finish = [&](int r, int c, int s, long long o, double a, double b, double e, double ku, double kv,
                      double kw) {
        const bool inner = (E == 0) || (r >= HALO && r < HALO + rows && c >= HALO && c < HALO + TX);
        const int d = (r - HALO) * TX + (c - HALO);
        if (MODE == 2) {
            const double nu = (a + D[d]) + cD * ku;
            out[o] = nu;
            out[g.plane + o] = (b + D[IN + d]) + cD * kv;
            out[2 * g.plane + o] = (e + D[2 * IN + d]) + cD * kw;
            const double t = nu * __ldg(gh + o);
            D[d] = isnan(t) ? 0.0 : t;
        } else {
            dst[s] = a + cZ * ku;
            dst[RN + s] = b + cZ * kv;
            dst[2 * RN + s] = e + cZ * kw;
            if (inner) {
                if (MODE == 0) {
                    D[d] = cD * ku;
                    D[IN + d] = cD * kv;
                    D[2 * IN + d] = cD * kw;
                } else {
                    D[d] = D[d] + cD * ku;
                    D[IN + d] = D[IN + d] + cD * kv;
                    D[2 * IN + d] = D[2 * IN + d] + cD * kw;
                }
            }
        }
    };
    RowCol<W, NT> rc(HALO - E, HALO - E);
    if constexpr (PF) {
        // Software-pipelined (the single-instance kernel): the next cell's
        // global operands (step-start state, weight code, cached Jacobian or
        // the state it is evaluated at) are loaded while this cell computes.
        struct Ops {
            double a, b, e, j[7];
            int code;
        };
        auto fetch = [&](int r, int c, Ops& x) {
            const long long o = off + (long long)r * g.ld + c;
            if (MODE != 0) x.a = __ldg(z0g + o), x.b = __ldg(z0g + g.plane + o), x.e = __ldg(z0g + 2 * g.plane + o);
            x.code = __ldg(wc + o);
            if (jload) {
#pragma unroll
                for (int k = 0; k < 7; ++k) x.j[k] = __ldg(jload + k * g.plane + o);
            } else {
                x.j[0] = __ldg(ys + o), x.j[1] = __ldg(ys + g.plane + o), x.j[2] = __ldg(ys + 2 * g.plane + o);
            }
        };
        // FKADJ_ADJ_PREFETCH=2 loads two cells ahead
        constexpr int DEPTH = FKADJ_ADJ_PREFETCH >= 2 ? 2 : 1;
        RowCol<W, NT> ahead = rc;  // the cell DEPTH cells after rc's
        Ops cur, n1;
        if ((int)threadIdx.x < N) fetch(ahead.r, ahead.c, cur);
        ahead.next();
        if constexpr (DEPTH == 2) {
            if ((int)threadIdx.x + NT < N) fetch(ahead.r, ahead.c, n1);
            ahead.next();
        }
        for (int q = threadIdx.x; q < N; q += NT) {
            const int r = rc.r, c = rc.c;
            rc.next();
            Ops nxt;
            if (q + DEPTH * NT < N) fetch(ahead.r, ahead.c, nxt);
            ahead.next();
            const int s = r * RW + c;
            const long long o = off + (long long)r * g.ld + c;
            double a = cur.a, b = cur.b, e = cur.e;
            if (MODE == 0) a = src[s], b = src[RN + s], e = src[2 * RN + s];
            double ku, kv, kw;
            if (isnan(src[s])) {  // holes and the NaN ring: the result is NaN
                ku = kv = kw = src[s];
            } else {
                JacT J;
                if (jload) {
                    J = {cur.j[0], cur.j[1], cur.j[2], cur.j[3], cur.j[4], cur.j[5], cur.j[6]};
                } else {
                    J = fk_jacT(P, finite_u(cur.j[0]), cur.j[1], cur.j[2]);
                    if (jstore) store_jac(jstore, g.plane, o, J);
                }
                adj_at<RW, RN>(P, src, s, cur.code, J, ku, kv, kw);
            }
            finish(r, c, s, o, a, b, e, ku, kv, kw);
            if constexpr (DEPTH == 2) {
                cur = n1;
                n1 = nxt;
            } else {
                cur = nxt;
            }
        }
    } else {
#pragma unroll kStageUnroll
        for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
            const int r = rc.r, c = rc.c;
            const int s = r * RW + c;
            const long long o = off + (long long)r * g.ld + c;
            double a, b, e;
            if (MODE == 0) {  // the first stage's source region is z0 itself
                a = src[s], b = src[RN + s], e = src[2 * RN + s];
            } else {
                a = __ldg(z0g + o), b = __ldg(z0g + g.plane + o), e = __ldg(z0g + 2 * g.plane + o);
            }
            const int code = __ldg(wc + o);
            double ku, kv, kw;
#if FKADJ_HOLE_BRANCH
            if (isnan(src[s])) {  // holes and the NaN ring: the result is NaN
                ku = kv = kw = src[s];
            } else
#endif
            {
                JacT J;
                if (jload) {
                    J = load_jac(jload, g.plane, o);
                } else {
                    J = fk_jacT(P, finite_u(__ldg(ys + o)), __ldg(ys + g.plane + o), __ldg(ys + 2 * g.plane + o));
                    if (jstore) store_jac(jstore, g.plane, o, J);
                }
                adj_at<RW, RN>(P, src, s, code, J, ku, kv, kw);
            }
            finish(r, c, s, o, a, b, e, ku, kv, kw);
        }
    }
    if (MODE != 2) __syncthreads();
}

// One backward RK4 step of the reference adjoint: stage 1 uses y(t_i) = yb,
// stages 2-3 the midpoint yh, stage 4 y(t_{i-1}) = ya; the tile's 16x16
// sub-block sums of z_u . gh (NaN terms skipped, cu-G:1457-1483) go to `row`.
// Jacobian caches (null = evaluate): jb = J(y_i) left by the previous step's
// last stage, jh = J(yh) from k_adj_mid; J(y_{i-1}) is evaluated in the last
// stage and stored to ja for the next step.
template <int TX, int TY, int NT, bool BULK = false, bool PF = false>
__device__ __forceinline__ void adj_step_tile(const DevModel& P, const DevGrid& g, const double* __restrict__ z,
                                              double* __restrict__ zout, const double* __restrict__ yb,
                                              const double* __restrict__ yh, const double* __restrict__ ya,
                                              const uint8_t* __restrict__ wc, const double* __restrict__ gh,
                                              double* __restrict__ row, int nsbx, const double* __restrict__ jb,
                                              const double* __restrict__ jh, double* __restrict__ ja, int tbx,
                                              int tby, unsigned* fault = nullptr, uint32_t* phase = nullptr,
                                              int ty = TY, bool segments = false) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
    extern __shared__ double4 smem_raw[];
    double* A = reinterpret_cast<double*>(smem_raw);
    double* B = A + 3 * RN;
    double* D = B + 3 * RN;
    // On the row-segment lattice a tile has ty <= TY rows, cut at the grid's
    // edge; on the 16x16 sub-block lattice ty = TY and the tile keeps all TY
    // rows (rows past the edge are NaN ring or padding and sum to 0).
    const int i0 = tby * ty, j0 = tbx * TX;
    const int rows = segments ? min(ty, g.nrows - i0) : TY;
    const long long off = (long long)i0 * g.ld + j0;
    const bool vec_ok = ((g.ld | j0) & 1) == 0;
    if (!load_windows<RH, RW, NT, BULK>(A, z + off, nullptr, nullptr, g.ld, g.plane, vec_ok, rows + 2 * HALO,
                                        fault, nullptr, nullptr, phase))
        return;
    const double dt = P.dt;
    adj_stage<3, TX, TY, NT, 0, PF>(P, g, A, B, D, z, wc, yb, off, 0.5 * dt, 1.0 / 6.0 * dt, nullptr, gh, jb,
                                    nullptr, rows);
    adj_stage<2, TX, TY, NT, 1, PF>(P, g, B, A, D, z, wc, yh, off, 0.5 * dt, 2.0 / 6.0 * dt, nullptr, gh, jh,
                                    nullptr, rows);
    adj_stage<1, TX, TY, NT, 1, PF>(P, g, A, B, D, z, wc, yh, off, dt, 2.0 / 6.0 * dt, nullptr, gh, jh, nullptr,
                                    rows);
    adj_stage<0, TX, TY, NT, 2, PF>(P, g, B, A, D, z, wc, ya, off, 0.0, 1.0 / 6.0 * dt, zout, gh, nullptr, ja,
                                    rows);
    __syncthreads();
    if (segments)
        segment_sums<TX, NT>([&](int r, int c) { return D[r * TX + c]; }, row, i0, j0, nsbx, rows);
    else
        subblock_sums<TX, TY, NT>([&](int r, int c) { return D[r * TX + c]; }, row, i0, j0, nsbx);
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, min_blocks(TX, TY, NT))
    k_adj_step(DevModel P, DevGrid g, const double* __restrict__ z, double* __restrict__ zout,
               const double* __restrict__ yb, const double* __restrict__ yh, const double* __restrict__ ya,
               const uint8_t* __restrict__ wc, const double* __restrict__ gh, double* __restrict__ row, int nsbx,
               const double* __restrict__ jb, const double* __restrict__ jh, double* __restrict__ ja,
               unsigned* fault, int ty, int segments) {
    pdl_enter();
    exp_table_init();
    adj_step_tile<TX, TY, NT, true, FKADJ_ADJ_PREFETCH != 0>(P, g, z, zout, yb, yh, ya, wc, gh, row, nsbx, jb, jh,
                                                             ja, blockIdx.x, blockIdx.y, fault, nullptr, ty,
                                                             segments != 0);
}

// ------------------------------------------- fused reference-mode adjoint
//
// One backward step of the reference adjoint in one launch: the midpoint
// reconstruction of k_adj_mid and the four stages of k_adj_step, with the
// midpoint state and its Jacobian never leaving the CTA.  The tile's windows
// of z, y_{i-1} and y_i (tile + 4) arrive by bulk copies; y(1/3) is formed on
// the tile + 3 and f(y(1/3)) on the tile + 2, so yh covers the region stage 2
// reads; J_F(yh)^T is evaluated where stages 2 and 3 need it instead of being
// stored and reloaded (k_adj_mid writes 80 B/cell that k_adj_step reads about
// 2.3 times).  Every value is the same computation on the same inputs as in
// the split kernels (cu-G:1244-1301 then cu-G:1349-1427 in the order of
// cu-G:1885-1891), so the gradient does not depend on which path runs.
//
// Stage 1's J_F(y_i)^T comes from the cache jb left by the previous step's
// stage 4 (which stores J_F(y_{i-1})^T to ja), or, with jb null, is evaluated
// from the y_i window; with ja null nothing is stored.  fa / fb are f(y_{i-1})
// and f(y_i) where kept or carried (null: evaluated from the windows); fout
// receives the evaluated f(y_{i-1}) on the tile for the next step's fb.
//
// One stage on the tile grown by E cells, k_adj_step's algebra with the
// step-start state z0 read from its shared-memory window Zw; jac(r, c, o)
// returns J_F^T at window cell (r, c), global offset o (called for non-hole
// cells only).
template <int E, int TX, int TY, int NT, int MODE, class Jac>
__device__ __forceinline__ void fused_stage(const DevModel& P, const DevGrid& g, const double* __restrict__ src,
                                            double* __restrict__ dst, double* __restrict__ D,
                                            const double* __restrict__ Zw, const uint8_t* __restrict__ wc,
                                            long long off, double cZ, double cD, double* __restrict__ out,
                                            const double* __restrict__ gh, Jac jac) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
    constexpr int W = TX + 2 * E, H = TY + 2 * E, N = W * H;
    constexpr int IN = TX * TY;
    RowCol<W, NT> rc(HALO - E, HALO - E);
#pragma unroll kStageUnroll
    for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
        const int r = rc.r, c = rc.c;
        const int s = r * RW + c;
        const long long o = off + (long long)r * g.ld + c;
        const double a = Zw[s], b = Zw[RN + s], e = Zw[2 * RN + s];
        const int code = __ldg(wc + o);
        double ku, kv, kw;
#if FKADJ_HOLE_BRANCH
        if (isnan(src[s])) {  // holes and the NaN ring: the result is NaN
            ku = kv = kw = src[s];
        } else
#endif
        {
            const JacT J = jac(r, c, o);
            adj_at<RW, RN>(P, src, s, code, J, ku, kv, kw);
        }
        const bool inner = (E == 0) || (r >= HALO && r < HALO + TY && c >= HALO && c < HALO + TX);
        const int d = (r - HALO) * TX + (c - HALO);
        if (MODE == 2) {
            const double nu = (a + D[d]) + cD * ku;
            out[o] = nu;
            out[g.plane + o] = (b + D[IN + d]) + cD * kv;
            out[2 * g.plane + o] = (e + D[2 * IN + d]) + cD * kw;
            const double t = nu * __ldg(gh + o);
            D[d] = isnan(t) ? 0.0 : t;
        } else {
            dst[s] = a + cZ * ku;
            dst[RN + s] = b + cZ * kv;
            dst[2 * RN + s] = e + cZ * kw;
            if (inner) {
                if (MODE == 0) {
                    D[d] = cD * ku;
                    D[IN + d] = cD * kv;
                    D[2 * IN + d] = cD * kw;
                } else {
                    D[d] = D[d] + cD * ku;
                    D[IN + d] = D[IN + d] + cD * kv;
                    D[2 * IN + d] = D[2 * IN + d] + cD * kw;
                }
            }
        }
    }
    if (MODE != 2) __syncthreads();
}

// Shared memory of k_adj_fused: windows of z, y_{i-1}, y_i on the tile + 4,
// y(1/3) on the tile + 3, the quartic part of yh (then yh) on the tile + 2,
// and the stage accumulator (206 KB at 32x32, 219 KB at 64x16, 119 KB at 32x16).
template <int TX, int TY>
constexpr size_t fused_smem_bytes() {
    return sizeof(double) * (9 * (TX + 2 * HALO) * (TY + 2 * HALO) + 3 * (TX + 6) * (TY + 6) +
                             3 * (TX + 4) * (TY + 4) + 3 * TX * TY);
}

template <int TX, int TY, int NT>
__device__ __forceinline__ void adj_fused_tile(const DevModel& P, const DevGrid& g, const double* __restrict__ z,
                                               double* __restrict__ zout, const double* __restrict__ ya,
                                               const double* __restrict__ yb, const double* __restrict__ fa,
                                               const double* __restrict__ fb, double* __restrict__ fout,
                                               const uint8_t* __restrict__ wc, const double* __restrict__ gh,
                                               double Ea, double Eb, double E3, const HermiteW& hw,
                                               double* __restrict__ row, int nsbx, const double* __restrict__ jb,
                                               double* __restrict__ ja, int tbx, int tby, unsigned* fault,
                                               uint32_t* phase = nullptr) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;  // windows: tile + 4
    constexpr int W3 = TX + 6, RN3 = W3 * (TY + 6);                      // y(1/3): tile + 3
    constexpr int WQ = TX + 4, RNQ = WQ * (TY + 4);                      // quartic part / yh: tile + 2
    extern __shared__ double4 smem_raw[];
    double* Zw = reinterpret_cast<double*>(smem_raw);
    double* YA = Zw + 3 * RN;  // y_{i-1}; stage 2 writes its state here
    double* YB = YA + 3 * RN;  // y_i; stages 1 and 3 write their states here
    double* Y3 = YB + 3 * RN;
    double* Q = Y3 + 3 * RN3;
    double* D = Q + 3 * RNQ;
    const int i0 = tby * TY, j0 = tbx * TX;
    const long long off = (long long)i0 * g.ld + j0;  // window origin: logical (i0 - 4, j0 - 4)
    const bool vec_ok = ((g.ld | j0) & 1) == 0;
    if (!load_windows<RH, RW, NT, true>(Zw, z + off, YA, ya + off, g.ld, g.plane, vec_ok, RH, fault, YB, yb + off,
                                        phase))
        return;
    const double dt = P.dt;
    // y(1/3) (cubic Hermite) on the tile + 3 and the quartic part of yh on the tile + 2
    {
        constexpr int W = TX + 6;
        constexpr int N = W * (TY + 6);
        RowCol<W, NT> rc(1, 1);
#pragma unroll kStageUnroll
        for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
            const int r = rc.r, c = rc.c;
            const int s = r * RW + c;
            const long long o = off + (long long)r * g.ld + c;
            const double gg = __ldg(gh + o);
            double a0[3], a1[3];
            if (fa) {
                a0[0] = __ldg(fa + o);
                a0[1] = __ldg(fa + g.plane + o);
                a0[2] = __ldg(fa + 2 * g.plane + o);
            } else {
                rhs_at<RW, RN>(P, YA, s, Ea * gg, a0[0], a0[1], a0[2], g.fcode ? (int)__ldg(g.fcode + o) : -1);
            }
            if (fb) {
                a1[0] = __ldg(fb + o);
                a1[1] = __ldg(fb + g.plane + o);
                a1[2] = __ldg(fb + 2 * g.plane + o);
            } else {
                rhs_at<RW, RN>(P, YB, s, Eb * gg, a1[0], a1[1], a1[2], g.fcode ? (int)__ldg(g.fcode + o) : -1);
            }
            if (fout && r >= HALO && r < HALO + TY && c >= HALO && c < HALO + TX) {
                fout[o] = a0[0];
                fout[g.plane + o] = a0[1];
                fout[2 * g.plane + o] = a0[2];
            }
            const int s3 = (r - 1) * W3 + (c - 1);
            const bool qcell = r >= 2 && r < RH - 2 && c >= 2 && c < RW - 2;
            const int sq = (r - 2) * WQ + (c - 2);
#pragma unroll
            for (int f = 0; f < 3; ++f) {
                const double m0 = a0[f] * dt, m1 = a1[f] * dt;
                const double x0 = YA[f * RN + s], x1 = YB[f * RN + s];
                Y3[f * RN3 + s3] = ((hw.c3[0] * x0 + hw.c3[1] * m0) + hw.c3[2] * x1) + hw.c3[3] * m1;
                if (qcell) Q[f * RNQ + sq] = ((hw.c4[0] * x0 + hw.c4[1] * m0) + hw.c4[2] * x1) + hw.c4[3] * m1;
            }
        }
    }
    __syncthreads();
    // yh = quartic part + (27/64) dt f(y(1/3), E(t_{i-1} + dt/3)) on the tile + 2
    {
        constexpr int W = TX + 4;
        constexpr int N = W * (TY + 4);
        RowCol<W, NT> rc(2, 2);
#pragma unroll kStageUnroll
        for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
            const int r = rc.r, c = rc.c;
            const long long o = off + (long long)r * g.ld + c;
            const int s3 = (r - 1) * W3 + (c - 1);
            const int sq = (r - 2) * WQ + (c - 2);
            double m2[3];
            rhs_at<W3, RN3>(P, Y3, s3, E3 * __ldg(gh + o), m2[0], m2[1], m2[2],
                            g.fcode ? (int)__ldg(g.fcode + o) : -1);
#pragma unroll
            for (int f = 0; f < 3; ++f) Q[f * RNQ + sq] = Q[f * RNQ + sq] + hw.c2 * (m2[f] * dt);
        }
    }
    __syncthreads();
    // the four backward stages (k_adj_step's): J(y_i), J(yh), J(yh), J(y_{i-1})
    auto j_yb = [&](int r, int c, long long o) -> JacT {
        if (jb) return load_jac(jb, g.plane, o);
        const int s = r * RW + c;
        return fk_jacT(P, finite_u(YB[s]), YB[RN + s], YB[2 * RN + s]);
    };
    auto j_yh = [&](int r, int c, long long) -> JacT {
        const int sq = (r - 2) * WQ + (c - 2);
        return fk_jacT(P, Q[sq], Q[RNQ + sq], Q[2 * RNQ + sq]);
    };
    auto j_ya = [&](int, int, long long o) -> JacT {
        const JacT J = fk_jacT(P, finite_u(__ldg(ya + o)), __ldg(ya + g.plane + o), __ldg(ya + 2 * g.plane + o));
        if (ja) store_jac(ja, g.plane, o, J);
        return J;
    };
    fused_stage<3, TX, TY, NT, 0>(P, g, Zw, YB, D, Zw, wc, off, 0.5 * dt, 1.0 / 6.0 * dt, nullptr, gh, j_yb);
    fused_stage<2, TX, TY, NT, 1>(P, g, YB, YA, D, Zw, wc, off, 0.5 * dt, 2.0 / 6.0 * dt, nullptr, gh, j_yh);
    fused_stage<1, TX, TY, NT, 1>(P, g, YA, YB, D, Zw, wc, off, dt, 2.0 / 6.0 * dt, nullptr, gh, j_yh);
    fused_stage<0, TX, TY, NT, 2>(P, g, YB, YA, D, Zw, wc, off, 0.0, 1.0 / 6.0 * dt, zout, gh, j_ya);
    __syncthreads();
    subblock_sums<TX, TY, NT>([&](int r, int c) { return D[r * TX + c]; }, row, i0, j0, nsbx);
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 1)
    k_adj_fused(DevModel P, DevGrid g, const double* __restrict__ z, double* __restrict__ zout,
                const double* __restrict__ ya, const double* __restrict__ yb, const double* __restrict__ fa,
                const double* __restrict__ fb, double* __restrict__ fout, const uint8_t* __restrict__ wc,
                const double* __restrict__ gh, EStep E, HermiteW hw, double* __restrict__ row, int nsbx,
                const double* __restrict__ jb, double* __restrict__ ja, unsigned* fault) {
    pdl_enter();
    exp_table_init();
    adj_fused_tile<TX, TY, NT>(P, g, z, zout, ya, yb, fa, fb, fout, wc, gh, E.a(), E.b(), E.c(), hw, row, nsbx, jb,
                               ja, blockIdx.x, blockIdx.y, fault);
}

// ------------------------------------------------------ exact-mode adjoint
//
// Discrete adjoint of one RK4 step y_{s+1} = y_s + dt/6 (k1 + 2k2 + 2k3 + k4):
// with lambda = dJ/dy_{s+1} and g(a; Y) = L^T a + J_F(Y)^T a,
//   a4 = dt/6 lam,                 mu4 = g(a4; Y4)
//   a3 = dt/3 lam + dt   mu4,      mu3 = g(a3; Y3)
//   a2 = dt/3 lam + dt/2 mu3,      mu2 = g(a2; Y2)
//   a1 = dt/6 lam + dt/2 mu2,      mu1 = g(a1; y_s)
//   lam_s = lam + (mu4 + mu3 + mu2 + mu1)
// and the E sensitivities b.a1 (sample s), b.(a2 + a3) (half step s) and
// b.a4 (sample s+1), b = gh on u.  Same temporal blocking as the reference
// mode: a_s lives in shared memory on the tile grown by (4 - s) cells.
template <int E, int TX, int TY, int NT, int MODE, bool PF = false>
__device__ __forceinline__ void exact_stage(const DevModel& P, const DevGrid& g, const double* __restrict__ src,
                                            double* __restrict__ dst, double* __restrict__ D,
                                            const double* __restrict__ lamg, const uint8_t* __restrict__ wc,
                                            const double* __restrict__ ys, long long off, double cL, double cM,
                                            double* __restrict__ out, double* __restrict__ keep_u) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
    constexpr int W = TX + 2 * E, H = TY + 2 * E, N = W * H;
    constexpr int IN = TX * TY;
    // the stage update of cell (r, c) from its lambda and k
    auto finish = [&](int r, int c, int s, long long o, double la, double lb, double lc, double ku, double kv,
                      double kw) {
        const bool inner = (E == 0) || (r >= HALO && r < HALO + TY && c >= HALO && c < HALO + TX);
        const int d = (r - HALO) * TX + (c - HALO);
        if (MODE == 2) {
            out[o] = la + (D[d] + ku);
            out[g.plane + o] = lb + (D[IN + d] + kv);
            out[2 * g.plane + o] = lc + (D[2 * IN + d] + kw);
        } else {
            const double au = cL * la + cM * ku;
            dst[s] = au;
            dst[RN + s] = cL * lb + cM * kv;
            dst[2 * RN + s] = cL * lc + cM * kw;
            if (inner) {
                if (MODE == 0) {
                    D[d] = ku;
                    D[IN + d] = kv;
                    D[2 * IN + d] = kw;
                } else {
                    D[d] = D[d] + ku;
                    D[IN + d] = D[IN + d] + kv;
                    D[2 * IN + d] = D[2 * IN + d] + kw;
                }
                if (keep_u) keep_u[d] = au;
            }
        }
    };
    RowCol<W, NT> rc(HALO - E, HALO - E);
    if constexpr (PF) {
        // Software-pipelined (the single-instance kernel): the next cell's
        // state (for its Jacobian), lambda and weight code are loaded while
        // this cell computes.
        struct Ops {
            double y[3], l[3];
            int code;
        };
        auto fetch = [&](int r, int c, Ops& x) {
            const long long o = off + (long long)r * g.ld + c;
#pragma unroll
            for (int f = 0; f < 3; ++f) x.y[f] = __ldg(ys + f * g.plane + o), x.l[f] = __ldg(lamg + f * g.plane + o);
            x.code = __ldg(wc + o);
        };
        Ops cur;
        if ((int)threadIdx.x < N) fetch(rc.r, rc.c, cur);
        for (int q = threadIdx.x; q < N; q += NT) {
            const int r = rc.r, c = rc.c;
            rc.next();
            Ops nxt;
            if (q + NT < N) fetch(rc.r, rc.c, nxt);
            const int s = r * RW + c;
            const long long o = off + (long long)r * g.ld + c;
            double ku, kv, kw;
            if (isnan(src[s])) {  // holes and the NaN ring: the result is NaN
                ku = kv = kw = src[s];
            } else {
                const JacT J = fk_jacT(P, finite_u(cur.y[0]), cur.y[1], cur.y[2]);
                adj_at<RW, RN>(P, src, s, cur.code, J, ku, kv, kw);
            }
            finish(r, c, s, o, cur.l[0], cur.l[1], cur.l[2], ku, kv, kw);
            cur = nxt;
        }
    } else {
#pragma unroll kStageUnroll
        for (int q = threadIdx.x; q < N; q += NT, rc.next()) {
            const int r = rc.r, c = rc.c;
            const int s = r * RW + c;
            const long long o = off + (long long)r * g.ld + c;
            double ku, kv, kw;
#if FKADJ_HOLE_BRANCH
            if (isnan(src[s])) {  // holes and the NaN ring: the result is NaN
                ku = kv = kw = src[s];
            } else
#endif
            {
                const JacT J =
                    fk_jacT(P, finite_u(__ldg(ys + o)), __ldg(ys + g.plane + o), __ldg(ys + 2 * g.plane + o));
                adj_at<RW, RN>(P, src, s, __ldg(wc + o), J, ku, kv, kw);
            }
            const double la = __ldg(lamg + o), lb = __ldg(lamg + g.plane + o), lc = __ldg(lamg + 2 * g.plane + o);
            finish(r, c, s, o, la, lb, lc, ku, kv, kw);
        }
    }
    if (MODE != 2) __syncthreads();
}

// lam (state of lambda_{s+1}) -> lamout (lambda_s); y = y_s; stages = Y2, Y3,
// Y4 of step s (three consecutive states, written by k_fwd_step).
// 16x16 sub-block sums: r1 <- b.a1, r23 <- b.(a2 + a3), r4 <- b.a4.
template <int TX, int TY, int NT, bool BULK = false, bool PF = false>
__device__ __forceinline__ void adj_exact_tile(const DevModel& P, const DevGrid& g, const double* __restrict__ lam,
                                               double* __restrict__ lamout, const double* __restrict__ y,
                                               const double* __restrict__ stages, const uint8_t* __restrict__ wc,
                                               const double* __restrict__ gh, double* __restrict__ r1,
                                               double* __restrict__ r23, double* __restrict__ r4, int nsbx, int tbx,
                                               int tby, unsigned* fault = nullptr, uint32_t* phase = nullptr) {
    constexpr int RW = TX + 2 * HALO, RH = TY + 2 * HALO, RN = RW * RH;
    constexpr int IN = TX * TY;
    extern __shared__ double4 smem_raw[];
    double* A = reinterpret_cast<double*>(smem_raw);
    double* B = A + 3 * RN;
    double* D = B + 3 * RN;
    double* T3 = D + 3 * IN;  // a3_u on the tile
    const int i0 = tby * TY, j0 = tbx * TX;
    const long long off = (long long)i0 * g.ld + j0;
    const bool vec_ok = ((g.ld | j0) & 1) == 0;
    if (!load_windows<RH, RW, NT, BULK>(A, lam + off, nullptr, nullptr, g.ld, g.plane, vec_ok, RH, fault, nullptr,
                                        nullptr, phase))
        return;
    const double dt = P.dt;
    const double c6 = dt / 6.0, c3 = dt / 3.0, c2 = dt * 0.5;
#pragma unroll 2
    for (int q = threadIdx.x; q < 3 * RN; q += NT) A[q] = c6 * A[q];  // a4
    __syncthreads();
    const long long sst = 3 * g.plane;
    exact_stage<3, TX, TY, NT, 0, PF>(P, g, A, B, D, lam, wc, stages + 2 * sst, off, c3, dt, nullptr, T3);
    exact_stage<2, TX, TY, NT, 1, PF>(P, g, B, A, D, lam, wc, stages + sst, off, c3, c2, nullptr, nullptr);
    exact_stage<1, TX, TY, NT, 1, PF>(P, g, A, B, D, lam, wc, stages, off, c6, c2, nullptr, nullptr);
    exact_stage<0, TX, TY, NT, 2, PF>(P, g, B, A, D, lam, wc, y, off, 0.0, 0.0, lamout, nullptr);
    __syncthreads();
    // now A holds a2 and B holds a1 on the tile
    auto ghv = [&](int r, int c) { return __ldg(gh + off + (long long)(r + HALO) * g.ld + (c + HALO)); };
    auto z0 = [](double t) { return isnan(t) ? 0.0 : t; };
    subblock_sums<TX, TY, NT>([&](int r, int c) { return z0(B[(r + HALO) * RW + c + HALO] * ghv(r, c)); },
                              r1, i0, j0, nsbx);
    subblock_sums<TX, TY, NT>(
        [&](int r, int c) { return z0((A[(r + HALO) * RW + c + HALO] + T3[r * TX + c]) * ghv(r, c)); }, r23, i0,
        j0, nsbx);
    subblock_sums<TX, TY, NT>(
        [&](int r, int c) {
            return z0(c6 * __ldg(lam + off + (long long)(r + HALO) * g.ld + (c + HALO)) * ghv(r, c));
        },
        r4, i0, j0, nsbx);
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, min_blocks(TX, TY, NT))
    k_adj_exact(DevModel P, DevGrid g, const double* __restrict__ lam, double* __restrict__ lamout,
                const double* __restrict__ y, const double* __restrict__ stages, const uint8_t* __restrict__ wc,
                const double* __restrict__ gh, double* __restrict__ r1, double* __restrict__ r23,
                double* __restrict__ r4, int nsbx, unsigned* fault) {
    pdl_enter();
    exp_table_init();
    adj_exact_tile<TX, TY, NT, true, FKADJ_ADJ_PREFETCH != 0>(P, g, lam, lamout, y, stages, wc, gh, r1, r23, r4, nsbx,
                                                              blockIdx.x, blockIdx.y, fault);
}

// ---------------------------------------------------------------- batched
//
// The batched kernels hold more live state than the single-instance ones (the
// work-queue item, the tile loop) and want up to 128 registers; the engine runs
// them with presets of at most 512 threads (batch_preset), where the 768- and
// 384-thread presets would cap them at 80 registers and spill heavily.
// One launch per kernel kind and tick runs the tiles of every instance that
// has that kind of work this tick.  The tick's work queue is in device memory
// (one small copy per tick; kernel parameters stay a few bytes); a persistent
// grid of CTAs strides over the queue's tiles, each item owning a contiguous
// range of tile indices.
__device__ __forceinline__ int find_item(const BatchItem* items, int n, int tile) {
    int lo = 0, hi = n - 1;
    while (lo < hi) {  // last item whose first tile is <= tile
        const int mid = (lo + hi + 1) >> 1;
        if (items[mid].tile0 <= tile) lo = mid;
        else hi = mid - 1;
    }
    return lo;
}

// The queue a batched launch works on: by value, or from its device header.
struct QueueView {
    const BatchItem* items;
    int n, tiles;
    __device__ __forceinline__ explicit QueueView(const BatchQueue& q) {
        if (q.hdr) {
            n = q.hdr[0];
            tiles = q.hdr[1];
            items = q.items + q.hdr[2];
        } else {
            n = q.n;
            tiles = q.tiles;
            items = q.items;
        }
    }
    __device__ __forceinline__ const BatchItem& item(int tile) const { return items[find_item(items, n, tile)]; }
};

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, FKADJ_BATCH_MINB(TX, TY, NT))
    k_batch_fwd(const BatchInstance* __restrict__ inst, const BatchQueue t) {
    pdl_enter();
    exp_table_init();
    uint32_t phase = 0;  // bulk transfers of this CTA so far (the tile-copy barrier's phase)
    const QueueView q(t);
    for (int tile = blockIdx.x; tile < q.tiles; tile += gridDim.x) {
        const BatchItem& it = q.item(tile);
        const BatchInstance& I = inst[it.inst];
        const int local = tile - it.tile0, tbx = local % it.ntx, tby = local / it.ntx;
        __syncthreads();
        fwd_step_tile<TX, TY, NT, true>(I.P, I.g, it.a, it.out, I.gh, it.E0, it.E1, it.E2, it.stages, tbx, tby, TY,
                                        it.k1, I.fault, &phase);
    }
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, FKADJ_BATCH_MINB(TX, TY, NT))
    k_batch_mid(const BatchInstance* __restrict__ inst, const BatchQueue t, HermiteW hw) {
    pdl_enter();
    exp_table_init();
    uint32_t phase = 0;
    const QueueView q(t);
    for (int tile = blockIdx.x; tile < q.tiles; tile += gridDim.x) {
        const BatchItem& it = q.item(tile);
        const BatchInstance& I = inst[it.inst];
        const int local = tile - it.tile0, tbx = local % it.ntx, tby = local / it.ntx;
        __syncthreads();
        adj_mid_tile<TX, TY, NT, true>(I.P, I.g, it.a, it.b, I.gh, it.out, it.E0, it.E1, it.E2, hw, it.fin, it.fout,
                                       it.jh, tbx, tby, TY, it.fa, I.fault, &phase);
    }
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, FKADJ_BATCH_MINB(TX, TY, NT))
    k_batch_adj(const BatchInstance* __restrict__ inst, const BatchQueue t) {
    pdl_enter();
    exp_table_init();
    uint32_t phase = 0;
    const QueueView q(t);
    for (int tile = blockIdx.x; tile < q.tiles; tile += gridDim.x) {
        const BatchItem& it = q.item(tile);
        const BatchInstance& I = inst[it.inst];
        const int local = tile - it.tile0, tbx = local % it.ntx, tby = local / it.ntx;
        __syncthreads();
        if (it.kind == BATCH_ADJ_EXACT)
            adj_exact_tile<TX, TY, NT, true>(I.P, I.g, it.a, it.out, it.b, it.stages, I.wc, I.gh, it.row, it.row2,
                                             it.row3, I.nsbx, tbx, tby, I.fault, &phase);
        else
            adj_step_tile<TX, TY, NT, true>(I.P, I.g, it.a, it.out, it.b, it.c, it.d, I.wc, I.gh, it.row, I.nsbx,
                                            it.jb, it.jh, it.ja, tbx, tby, I.fault, &phase);
    }
}

template <int TX, int TY, int NT>
__global__ void __launch_bounds__(NT, 1) k_batch_fused(const BatchInstance* __restrict__ inst, const BatchQueue t,
                                                       HermiteW hw) {
    pdl_enter();
    exp_table_init();
    uint32_t phase = 0;
    const QueueView q(t);
    for (int tile = blockIdx.x; tile < q.tiles; tile += gridDim.x) {
        const BatchItem& it = q.item(tile);
        const BatchInstance& I = inst[it.inst];
        const int local = tile - it.tile0, tbx = local % it.ntx, tby = local / it.ntx;
        __syncthreads();
        adj_fused_tile<TX, TY, NT>(I.P, I.g, it.a, it.out, it.d, it.b, it.fa, it.fin, it.fout, I.wc, I.gh, it.E0,
                                   it.E1, it.E2, hw, it.row, I.nsbx, it.jb, it.ja, tbx, tby, I.fault, &phase);
    }
}

// z_u . gh per 16x16 sub-block (NaN terms skipped), one warp per sub-block,
// in the order of subblock_sums -> row[sub-block].
__global__ void __launch_bounds__(32) k_dot_gh(DevGrid g, const double* __restrict__ z,
                                               const double* __restrict__ gh, double* __restrict__ row,
                                               int nsbx) {
    const int b = blockIdx.x, by = b / nsbx, bx = b - by * nsbx;
    subblock_sums<16, 16, 32>(
        [&](int r, int c) {
            const long long o = (long long)(by * 16 + r + HALO) * g.ld + (bx * 16 + c + HALO);
            const double t = z[o] * gh[o];
            return isnan(t) ? 0.0 : t;
        },
        row, by * 16, bx * 16, nsbx);
}

// The same on the row-segment lattice (segment_sums' order): half-warp h of
// block b takes segment 16 b + h of the grid (nseg = nsbx x nrows, row-major).
__global__ void __launch_bounds__(256) k_dot_gh_segments(DevGrid g, const double* __restrict__ z,
                                                         const double* __restrict__ gh, double* __restrict__ row,
                                                         int nsbx, int nseg) {
    const int l = threadIdx.x & 15;
    const int b = blockIdx.x * 16 + (threadIdx.x >> 4);
    const bool on = b < nseg;
    const int r = on ? b / nsbx : 0, sx = on ? b - r * nsbx : 0;
    double s = 0.0;
    if (on) {
        const long long o = (long long)(r + HALO) * g.ld + (sx * 16 + l + HALO);
        const double t = z[o] * gh[o];
        s = isnan(t) ? 0.0 : t;
    }
#pragma unroll
    for (int o = 8; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
    if (on && l == 0) row[b] = s;
}

// out[row] = sum_k partial[row*ntiles + k], fixed order (one block per row).
__global__ void k_sum_rows(const double* __restrict__ partial, int ntiles, double* __restrict__ out) {
    __shared__ double red[8];
    const double* p = partial + (long long)blockIdx.x * ntiles;
    double acc = 0.0;
    for (int k = threadIdx.x; k < ntiles; k += 256) acc += p[k];
    const double s = block_sum<256>(acc, red);
    if (threadIdx.x == 0) out[blockIdx.x] = s;
}

// ----------------------------------------------------------- layout kernels

// Compact [u;v;w] (n_num each, scaled by `scale`) -> padded NaN grid.
__global__ void k_scatter(DevGrid g, const double* __restrict__ yc, int n_num,
                          const long long* __restrict__ pos, double scale, double* __restrict__ y) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_num) return;
    const long long o = pos[m];
    y[o] = yc[m] * scale;
    y[g.plane + o] = yc[n_num + m] * scale;
    y[2 * g.plane + o] = yc[2 * n_num + m] * scale;
}

// Padded grid -> compact [u;v;w].
__global__ void k_gather(DevGrid g, const double* __restrict__ y, int n_num,
                         const long long* __restrict__ pos, double* __restrict__ yc) {
    const int m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= n_num) return;
    const long long o = pos[m];
    yc[m] = y[o];
    yc[n_num + m] = y[g.plane + o];
    yc[2 * n_num + m] = y[2 * g.plane + o];
}

// Objective at T: for each field f, zc_f = -gamma_f * (S y_f) with S in CSR
// (row sums in ascending column order, the order of the reference's CSC
// accumulation, cu-G:1514-1522); per-block partials of y_f . zc_f.
__global__ void k_objective(const double* __restrict__ yc, int n_num, const long long* __restrict__ rowptr,
                            const int* __restrict__ colidx, const double* __restrict__ val, double g0,
                            double g1, double g2, double* __restrict__ zc, double* __restrict__ partial) {
    __shared__ double red[8];
    const int r = blockIdx.x * 256 + threadIdx.x;
    double acc = 0.0;
    if (r < n_num) {
        double s0 = 0.0, s1 = 0.0, s2 = 0.0;
        for (long long k = rowptr[r]; k < rowptr[r + 1]; ++k) {
            const int c = colidx[k];
            const double a = val[k];
            s0 += a * yc[c];
            s1 += a * yc[n_num + c];
            s2 += a * yc[2 * n_num + c];
        }
        const double z0 = s0 * -g0, z1 = s1 * -g1, z2 = s2 * -g2;
        zc[r] = z0;
        zc[n_num + r] = z1;
        zc[2 * n_num + r] = z2;
        acc = (yc[r] * z0 + yc[n_num + r] * z1) + yc[2 * n_num + r] * z2;
    }
    const double s = block_sum<256>(acc, red);
    if (threadIdx.x == 0) partial[blockIdx.x] = s;
}

}  // namespace

// --------------------------------------------------------------- launchers

// two 3-field region buffers + the 3-field interior accumulator; the exact
// adjoint keeps one more interior plane (a3_u)
template <int TX, int TY>
static size_t stencil_smem(int /*nt*/) {
    constexpr int RN = (TX + 2 * HALO) * (TY + 2 * HALO);
    return sizeof(double) * (6 * RN + 3 * TX * TY);
}
template <int TX, int TY>
static size_t exact_smem() {
    constexpr int RN = (TX + 2 * HALO) * (TY + 2 * HALO);
    return sizeof(double) * (6 * RN + 4 * TX * TY);
}
// windows of y_{i-1}, y_i and y(1/3) on the tile + 2, and the quartic part of
// yh on the tile (225 KB at 64x32)
template <int TX, int TY>
static size_t mid_smem() {
    constexpr int RN = (TX + 4) * (TY + 4);
    return sizeof(double) * (9 * RN + 3 * TX * TY);
}

template <int TX, int TY, int NT>
static cudaError_t setup_tile() {
    cudaError_t e;
    const int s = (int)stencil_smem<TX, TY>(NT);
    if ((e = cudaFuncSetAttribute(k_fwd_step<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s))) return e;
    if ((e = cudaFuncSetAttribute(k_adj_step<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s))) return e;
    if ((e = cudaFuncSetAttribute(k_adj_exact<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)exact_smem<TX, TY>())))
        return e;
    if ((e = cudaFuncSetAttribute(k_batch_fwd<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, s))) return e;
    if ((e = cudaFuncSetAttribute(k_batch_mid<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)mid_smem<TX, TY>())))
        return e;
    if ((e = cudaFuncSetAttribute(k_batch_adj<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                  (int)exact_smem<TX, TY>())))
        return e;
    return cudaFuncSetAttribute(k_adj_mid<TX, TY, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                (int)mid_smem<TX, TY>());
}

// Persistent grid for a batched launch: as many CTAs as fit on the device at
// once (occupancy x SMs), never more than the tick's tiles.
template <class K>
static int persistent_grid(K kernel, int nt, size_t smem, int tiles) {
    static thread_local int sms = 0;
    if (!sms) {
        int dev = 0;
        cudaGetDevice(&dev);
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
        if (sms <= 0) sms = 1;
    }
    // occupancy per kernel, computed once (a per-tick query costs host time)
    static thread_local std::vector<std::pair<const void*, int>> occ;
    int per_sm = 0;
    for (auto& o : occ)
        if (o.first == (const void*)kernel) per_sm = o.second;
    if (per_sm == 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nt, smem) != cudaSuccess || per_sm < 1)
            per_sm = 1;
        occ.push_back({(const void*)kernel, per_sm});
    }
    const int g = sms * per_sm;
    return tiles < g ? tiles : g;
}

// Tile presets (TX, TY, threads).  All TY divide 64 (the row padding of the
// state planes) and all TX are multiples of 16.
#define FKADJ_TILE_LIST(X) \
    X(0, 32, 32, 256)      \
    X(1, 32, 32, 512)      \
    X(2, 64, 32, 512)      \
    X(3, 32, 16, 256)      \
    X(4, 16, 16, 256)      \
    X(5, 64, 16, 512)      \
    X(6, 64, 32, 768)      \
    X(7, 32, 32, 384)      \
    X(8, 64, 32, 640)

int tile_count() { return 9; }

int batch_preset(int t) {
    // 64x32/768 and /640 -> 64x32/512, 32x32/384 -> 32x32/512: more threads per CTA would
    // cap the batched kernels below the registers they need
    if (t == 6 || t == 8) return 2;
    if (t == 7) return 1;
    return t;
}

TileShape tile_shape(int t) {
    switch (t) {
#define X(id, a, b, c) \
    case id: return {a, b, c};
        FKADJ_TILE_LIST(X)
#undef X
        default: return {32, 32, 256};
    }
}

cudaError_t take_device_fault(cudaStream_t st, unsigned* d_fault, unsigned* fault) {
    unsigned v = 0;
    cudaError_t e = cudaMemcpyAsync(&v, d_fault, sizeof v, cudaMemcpyDeviceToHost, st);
    if (!e) e = cudaStreamSynchronize(st);
    if (!e && v) {
        e = cudaMemsetAsync(d_fault, 0, sizeof v, st);
        if (!e) e = cudaStreamSynchronize(st);
    }
    *fault = v;
    return e;
}

// Tile presets of the fused reference adjoint (TX, TY, threads): TX divides
// 64 (the padding of a state row: wider tiles would run past the row), TY a
// multiple of 16 that divides 64 (the z.gh sub-block sums, the row padding).
#define FKADJ_FUSED_LIST(X) \
    X(0, 32, 32, 512)       \
    X(1, 64, 16, 512)       \
    X(2, 32, 32, 384)       \
    X(3, 32, 16, 256)

int fused_count() { return 4; }

TileShape fused_shape(int t) {
    switch (t) {
#define X(id, a, b, c) \
    case id: return {a, b, c};
        FKADJ_FUSED_LIST(X)
#undef X
        default: return {32, 32, 512};
    }
}

cudaError_t kernels_init() {
    cudaError_t e;
#define X(id, a, b, c) \
    if ((e = setup_tile<a, b, c>()) != cudaSuccess) return e;
    FKADJ_TILE_LIST(X)
#undef X
#define X(id, a, b, c)                                                                                  \
    if ((e = cudaFuncSetAttribute(k_adj_fused<a, b, c>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)fused_smem_bytes<a, b>())) != cudaSuccess)                        \
        return e;                                                                                        \
    if ((e = cudaFuncSetAttribute(k_batch_fused<a, b, c>, cudaFuncAttributeMaxDynamicSharedMemorySize, \
                                  (int)fused_smem_bytes<a, b>())) != cudaSuccess)                        \
        return e;
    FKADJ_FUSED_LIST(X)
#undef X
    return cudaSuccess;
}


// Launches a step kernel with programmatic stream serialisation (the kernel
// starts with pdl_enter()).  FKADJ_NO_PDL=1 in the environment launches them
// plainly (pdl_enter then returns at once), and so does a thread that is
// capturing a graph (set_launch_pdl(false)): measured on B200, the attribute
// shortens the gaps between plain launches (134 -> 127 ms per 512^2 x 2000
// gradient) but lengthens a replayed graph (37 -> 44 ms at 128^2).
static thread_local bool t_pdl_on = true;
void set_launch_pdl(bool on) { t_pdl_on = on; }
static bool pdl_enabled() {
    static const bool env_on = [] {
        const char* v = getenv("FKADJ_NO_PDL");
        return !(v && v[0] && v[0] != '0');
    }();
    return env_on && t_pdl_on;
}

template <typename... KArgs, typename... Args>
static cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, int threads, size_t smem, cudaStream_t st,
                              Args&&... args) {
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = dim3(threads);
    cfg.dynamicSmemBytes = smem;
    cfg.stream = st;
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cfg.attrs = at;
    cfg.numAttrs = pdl_enabled() ? 1 : 0;
    return cudaLaunchKernelEx(&cfg, kernel, std::forward<Args>(args)...);
}

#define DISPATCH(tile, ...)                               \
    switch (tile) {                                       \
        case 1: { constexpr int TX = 32, TY = 32, NT = 512; __VA_ARGS__; } break; \
        case 2: { constexpr int TX = 64, TY = 32, NT = 512; __VA_ARGS__; } break; \
        case 3: { constexpr int TX = 32, TY = 16, NT = 256; __VA_ARGS__; } break; \
        case 4: { constexpr int TX = 16, TY = 16, NT = 256; __VA_ARGS__; } break; \
        case 5: { constexpr int TX = 64, TY = 16, NT = 512; __VA_ARGS__; } break; \
        case 6: { constexpr int TX = 64, TY = 32, NT = 768; __VA_ARGS__; } break; \
        case 7: { constexpr int TX = 32, TY = 32, NT = 384; __VA_ARGS__; } break; \
        case 8: { constexpr int TX = 64, TY = 32, NT = 640; __VA_ARGS__; } break; \
        default: { constexpr int TX = 32, TY = 32, NT = 256; __VA_ARGS__; } break; \
    }

static dim3 tile_grid(const DevGrid& g, int tx, int ty) {
    return dim3((g.ncols + tx - 1) / tx, (g.nrows + ty - 1) / ty);
}

cudaError_t launch_fwd_step(int tile, const DevModel& P, const DevGrid& g, const double* yin, double* yout,
                            const double* gh, const EStep& E, cudaStream_t st, unsigned* fault, double* stages, int ty,
                            double* k1) {
    DISPATCH(tile, {
        const int rows = (ty > 0 && ty < TY) ? ty : TY;
        const cudaError_t e = launch_pdl(k_fwd_step<TX, TY, NT>, tile_grid(g, TX, rows), NT,
                                         stencil_smem<TX, TY>(NT), st, P, g, yin, yout, gh, E, stages, rows, k1, fault);
        if (e != cudaSuccess) return e;
    });
    return cudaGetLastError();
}

cudaError_t launch_adj_exact(int tile, const DevModel& P, const DevGrid& g, const double* lam, double* lamout,
                             const double* y, const double* stages, const uint8_t* wc, const double* gh,
                             double* r1, double* r23, double* r4, int nsbx, cudaStream_t st, unsigned* fault) {
    DISPATCH(tile, {
        const cudaError_t e = launch_pdl(k_adj_exact<TX, TY, NT>, tile_grid(g, TX, TY), NT, exact_smem<TX, TY>(), st,
                                         P, g, lam, lamout, y, stages, wc, gh, r1, r23, r4, nsbx, fault);
        if (e != cudaSuccess) return e;
    });
    return cudaGetLastError();
}

cudaError_t launch_adj_mid(int tile, const DevModel& P, const DevGrid& g, const double* ya, const double* yb,
                           const double* gh, double* yh, const EStep& E, const HermiteW& hw, cudaStream_t st,
                           unsigned* fault, const double* fin, double* fout, double* jh, int ty, const double* fa) {
    DISPATCH(tile, {
        const int rows = (ty > 0 && ty < TY) ? ty : TY;
        const cudaError_t e = launch_pdl(k_adj_mid<TX, TY, NT>, tile_grid(g, TX, rows), NT, mid_smem<TX, TY>(), st,
                                         P, g, ya, yb, gh, yh, E, hw, fin, fout, jh, rows, fa, fault);
        if (e != cudaSuccess) return e;
    });
    return cudaGetLastError();
}

// Rows per tile that spread the grid over one wave of CTAs (occupancy x SMs)
// with as little work per CTA as the preset's width allows; the preset's own
// height when the grid needs more than one wave at that height.
template <class K>
static int wave_rows(K kernel, int nt, size_t smem, int tx, int ty, const DevGrid& g) {
    int dev = 0, sms = 0, per_sm = 0;
    if (cudaGetDevice(&dev) != cudaSuccess ||
        cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return ty;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, nt, smem) != cudaSuccess || per_sm < 1)
        return ty;
    const int ntx = (g.ncols + tx - 1) / tx;
    const int nty = (sms * per_sm) / ntx;
    if (nty < 1) return ty;
    const int rows = (g.nrows + nty - 1) / nty;
    return rows < ty ? rows : ty;
}

int balanced_rows(int tile, int kind, const DevGrid& g) {
    int r = 0;
    DISPATCH(tile, {
        r = kind == 0   ? wave_rows(k_fwd_step<TX, TY, NT>, NT, stencil_smem<TX, TY>(NT), TX, TY, g)
            : kind == 1 ? wave_rows(k_adj_mid<TX, TY, NT>, NT, mid_smem<TX, TY>(), TX, TY, g)
                        : wave_rows(k_adj_step<TX, TY, NT>, NT, stencil_smem<TX, TY>(NT), TX, TY, g);
    });
    return r;
}

cudaError_t launch_adj_step(int tile, const DevModel& P, const DevGrid& g, const double* z, double* zout,
                            const double* yb, const double* yh, const double* ya, const uint8_t* wc,
                            const double* gh, double* row, int nsbx, cudaStream_t st, unsigned* fault,
                            const double* jb, const double* jh, double* ja, int ty, bool segments) {
    DISPATCH(tile, {
        // rows other than the preset's height only on the row-segment lattice
        const int rows = (segments && ty > 0 && ty < TY) ? ty : TY;
        const cudaError_t e = launch_pdl(k_adj_step<TX, TY, NT>, tile_grid(g, TX, rows), NT, stencil_smem<TX, TY>(NT),
                                         st, P, g, z, zout, yb, yh, ya, wc, gh, row, nsbx, jb, jh, ja, fault, rows,
                                         segments ? 1 : 0);
        if (e != cudaSuccess) return e;
    });
    return cudaGetLastError();
}

cudaError_t launch_adj_fused(int tile, const DevModel& P, const DevGrid& g, const double* z, double* zout,
                             const double* ya, const double* yb, const double* fa, const double* fb, double* fout,
                             const uint8_t* wc, const double* gh, const EStep& E, const HermiteW& hw, double* row,
                             int nsbx, const double* jb, double* ja, cudaStream_t st, unsigned* fault) {
    switch (tile) {
#define X(id, a, b, c)                                                                                        \
    case id: {                                                                                                \
        const cudaError_t e = launch_pdl(k_adj_fused<a, b, c>, tile_grid(g, a, b), c, fused_smem_bytes<a, b>(), \
                                         st, P, g, z, zout, ya, yb, fa, fb, fout, wc, gh, E, hw, row, nsbx, jb,  \
                                         ja, fault);                                                           \
        if (e != cudaSuccess) return e;                                                                       \
    } break;
        FKADJ_FUSED_LIST(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

// A launch whose queue is read from its device header (t.hdr) takes the full
// persistent grid: the number of tiles is not known on the host.
static int queue_tiles(const BatchQueue& t) { return t.hdr ? (1 << 30) : t.tiles; }

cudaError_t launch_batch_fwd(int tile, const BatchInstance* d_inst, const BatchQueue& t, cudaStream_t st) {
    if (!t.hdr && (t.n <= 0 || t.tiles <= 0)) return cudaSuccess;
    DISPATCH(tile, {
        const size_t sm = stencil_smem<TX, TY>(NT);
        const int grid = persistent_grid(k_batch_fwd<TX, TY, NT>, NT, sm, queue_tiles(t));
        const cudaError_t e = launch_pdl(k_batch_fwd<TX, TY, NT>, dim3(grid), NT, sm, st, d_inst, t);
        if (e != cudaSuccess) return e;
    });
    return cudaGetLastError();
}

cudaError_t launch_batch_mid(int tile, const BatchInstance* d_inst, const BatchQueue& t, const HermiteW& hw,
                             cudaStream_t st) {
    if (!t.hdr && (t.n <= 0 || t.tiles <= 0)) return cudaSuccess;
    DISPATCH(tile, {
        const size_t sm = mid_smem<TX, TY>();
        const int grid = persistent_grid(k_batch_mid<TX, TY, NT>, NT, sm, queue_tiles(t));
        const cudaError_t e = launch_pdl(k_batch_mid<TX, TY, NT>, dim3(grid), NT, sm, st, d_inst, t, hw);
        if (e != cudaSuccess) return e;
    });
    return cudaGetLastError();
}

cudaError_t launch_batch_adj(int tile, const BatchInstance* d_inst, const BatchQueue& t, cudaStream_t st) {
    if (!t.hdr && (t.n <= 0 || t.tiles <= 0)) return cudaSuccess;
    DISPATCH(tile, {
        const size_t sm = exact_smem<TX, TY>();
        const int grid = persistent_grid(k_batch_adj<TX, TY, NT>, NT, sm, queue_tiles(t));
        const cudaError_t e = launch_pdl(k_batch_adj<TX, TY, NT>, dim3(grid), NT, sm, st, d_inst, t);
        if (e != cudaSuccess) return e;
    });
    return cudaGetLastError();
}

cudaError_t launch_batch_fused(int tile, const BatchInstance* d_inst, const BatchQueue& t, const HermiteW& hw,
                               cudaStream_t st) {
    if (!t.hdr && (t.n <= 0 || t.tiles <= 0)) return cudaSuccess;
    switch (tile) {
#define X(id, a, b, c)                                                                                  \
    case id: {                                                                                          \
        const size_t sm = fused_smem_bytes<a, b>();                                                      \
        const int grid = persistent_grid(k_batch_fused<a, b, c>, c, sm, queue_tiles(t));                 \
        const cudaError_t e = launch_pdl(k_batch_fused<a, b, c>, dim3(grid), c, sm, st, d_inst, t, hw); \
        if (e != cudaSuccess) return e;                                                                 \
    } break;
        FKADJ_FUSED_LIST(X)
#undef X
        default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

cudaError_t launch_dot_gh(const DevGrid& g, const double* z, const double* gh, double* row, int nsbx, int nsby,
                          cudaStream_t st, bool segments) {
    if (segments) {
        const int nseg = nsbx * g.nrows;
        k_dot_gh_segments<<<(nseg + 15) / 16, 256, 0, st>>>(g, z, gh, row, nsbx, nseg);
    } else {
        k_dot_gh<<<nsbx * nsby, 32, 0, st>>>(g, z, gh, row, nsbx);
    }
    return cudaGetLastError();
}

void subblock_lattice(const DevGrid& g, int* nsbx, int* nsby) {
    *nsbx = ((g.ncols + 63) / 64) * 4;
    *nsby = ((g.nrows + 63) / 64) * 4;
}

int tiles_of(int tile, const DevGrid& g) {
    const TileShape t = tile_shape(tile);
    return ((g.ncols + t.tx - 1) / t.tx) * ((g.nrows + t.ty - 1) / t.ty);
}

cudaError_t launch_sum_rows(const double* partial, int rows, int ntiles, double* out, cudaStream_t st) {
    if (rows <= 0) return cudaSuccess;
    k_sum_rows<<<rows, 256, 0, st>>>(partial, ntiles, out);
    return cudaGetLastError();
}

cudaError_t launch_scatter(const DevGrid& g, const double* yc, int n_num, const long long* pos, double scale,
                           double* y, cudaStream_t st) {
    k_scatter<<<(n_num + 255) / 256, 256, 0, st>>>(g, yc, n_num, pos, scale, y);
    return cudaGetLastError();
}

cudaError_t launch_gather(const DevGrid& g, const double* y, int n_num, const long long* pos, double* yc,
                          cudaStream_t st) {
    k_gather<<<(n_num + 255) / 256, 256, 0, st>>>(g, y, n_num, pos, yc);
    return cudaGetLastError();
}

int objective_blocks(int n_num) { return (n_num + 255) / 256; }

cudaError_t launch_objective(const double* yc, int n_num, const long long* rowptr, const int* colidx,
                             const double* val, const double gamma[3], double* zc, double* partial,
                             cudaStream_t st) {
    k_objective<<<objective_blocks(n_num), 256, 0, st>>>(yc, n_num, rowptr, colidx, val, gamma[0], gamma[1],
                                                         gamma[2], zc, partial);
    return cudaGetLastError();
}

}  // namespace fkadj
