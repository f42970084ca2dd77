// sp_kernels_x2.cuh — the FP32 step kernel with two particles per thread in paired
// (f32x2) arithmetic, for the Brown+Neel Euler/spherical problem and its explicit
// steppers (EulerMaruyama, Heun, Millstein, EulerMaruyama_Normalized).
//
// Thread t of a tile integrates particles first + t (lane x) and first + blockDim + t
// (lane y) with the physics of sp_physics.cuh instantiated on F2 (sp_pack.cuh), so every
// add, multiply and fused multiply-add of the drift, diffusion, stepper and window sums
// covers both particles in one instruction; Philox, Box-Muller and the sines and cosines
// run per lane.  Each particle's chart (Euler and Neel coordinate rotations near a pole,
// BrownAndNeelRelaxationEulerSpherical.h:141-361) is decided per lane: when both lanes
// share their charts one pass advances both; otherwise the step runs once per lane's
// chart pair and each lane keeps the pass made in its own charts, so a particle's
// arithmetic never depends on its partner.  The passes are one inlined copy of the step
// in a loop (a called routine would take the addresses of the state and the prefactors
// and keep them in local memory on every step).
#pragma once

#include "sp_kernels.cuh"
#include "sp_pack.cuh"

namespace sp {

template <int PROB, int A, int SOLVER>
__global__ void __launch_bounds__(kMaxBlock / 2) step_kernel_x2(const EnsDev* __restrict__ ensembles,
                                                                const TileDesc* __restrict__ tiles, int ntiles) {
    using PX = typename ProblemOf<PROB, F2, A>::type;
    using St = Stepper<PX, F2, SOLVER>;
    static_assert(St::kExplicit, "the paired kernel covers the explicit steppers");
    constexpr int D = PX::D, Mn = PX::Mn, OUT = PX::OUT;
    // per-warp copy of the chunk's field table, each value in both lanes
    __shared__ float2 sBw[kMaxBlock / 64][kFieldTile][3];
    float2(*const sB)[3] = sBw[threadIdx.x >> 5];

    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const TileDesc td = tiles[t];
        const EnsDev& e = ensembles[td.ens];
        const unsigned long long s0 = e.ctl->step_done, tgt = e.ctl->step_target;
        const unsigned long long nsteps = tgt > s0 ? min(e.chunk, tgt - s0) : 0ull;
        if (nsteps == 0) continue;  // uniform across the CTA
        const unsigned long long Np = e.Np, W = e.W;
        const unsigned long long p[2] = {td.first + threadIdx.x, td.first + blockDim.x + threadIdx.x};
        const bool active[2] = {p[0] < e.n, p[1] < e.n};
        // an idle lane repeats the thread's other particle (or the tile's first), so it
        // takes the same charts and its results are discarded
        const unsigned long long src0 = active[0] ? p[0] : td.first, src1 = active[1] ? p[1] : src0;
        const float dt1 = static_cast<float>(e.dt);
        const F2 dt(dt1);
        const float sqdt = static_cast<float>(e.sqrt_dt), m2dt = static_cast<float>(-2.0 * e.dt);
        const unsigned long long seed = e.seed;
        const float* ftab = static_cast<const float*>(e.ftab);
        const bool rb = e.rot_brown != 0, rn = e.rot_neel != 0;
        const float min1 = static_cast<float>(e.min1), max1 = static_cast<float>(e.max1);
        const float min2 = static_cast<float>(e.min2), max2 = static_cast<float>(e.max2);

        const float* state = static_cast<const float*>(e.state);
        const float* ks = static_cast<const float*>(e.ksum);
        const float* kc = static_cast<const float*>(e.kcomp);
        const float* prm = static_cast<const float*>(e.params);
        F2 y[D];
#pragma unroll
        for (int i = 0; i < D; ++i) y[i] = F2(state[i * Np + src0], state[i * Np + src1]);
        WindowSum<F2, OUT> acc;
#pragma unroll
        for (int c = 0; c < OUT; ++c)
            acc.set(c, F2(ks[c * Np + src0], ks[c * Np + src1]), F2(kc[c * Np + src0], kc[c * Np + src1]));
        const typename PX::Par q = PX::load_with([&](int i) { return F2(prm[i * Np + src0], prm[i * Np + src1]); });
        typename PX::Trig tr;
        PX::trig(y, tr);
        const Rot<F2> rot{};

        unsigned int wpos = static_cast<unsigned int>(s0 % W);
        const unsigned int W32 = static_cast<unsigned int>(W);
        for (unsigned long long t0 = 0; t0 < nsteps; t0 += kFieldTile) {
            const int len = static_cast<int>(min(static_cast<unsigned long long>(kFieldTile), nsteps - t0));
            __syncwarp();
            for (int i = threadIdx.x & 31; i < 3 * len; i += 32) {
                const float b = ftab[3 * t0 + i];
                (&sB[0][0])[i] = make_float2(b, b);
            }
            __syncwarp();
            for (int i = 0; i < len; ++i) {
                const unsigned long long g = s0 + t0 + i;
                const F2 B[3] = {F2(sB[i][0]), F2(sB[i][1]), F2(sB[i][2])};
                float w0[Mn], w1[Mn];
                philox_increments<float, Mn, PX::kCalledMath>(seed, e.pid_offset + src0, g, sqdt, m2dt, w0);
                if (active[1]) {
                    philox_increments<float, Mn, PX::kCalledMath>(seed, e.pid_offset + p[1], g, sqdt, m2dt, w1);
                } else {
#pragma unroll
                    for (int j = 0; j < Mn; ++j) w1[j] = w0[j];
                }
                F2 w[Mn];
#pragma unroll
                for (int j = 0; j < Mn; ++j) w[j] = F2(w0[j], w1[j]);
                // charts of each lane (prepareCalculations, :141-150)
                const float tb0 = fabsf(lane0(y[1])), tb1 = fabsf(lane1(y[1]));
                const float tn0 = fabsf(lane0(y[3])), tn1 = fabsf(lane1(y[3]));
                const bool br0 = rb && (tb0 < min1 || tb0 > max1), br1 = rb && (tb1 < min1 || tb1 > max1);
                const bool nr0 = rn && (tn0 < min2 || tn0 > max2), nr1 = rn && (tn1 < min2 || tn1 > max2);
                const int passes = (br0 == br1 && nr0 == nr1) ? 1 : 2;
                F2 y0[D];
#pragma unroll
                for (int d = 0; d < D; ++d) y0[d] = y[d];
#pragma unroll 1
                for (int pass = 0; pass < passes; ++pass) {
                    F2 yp[D];
#pragma unroll
                    for (int d = 0; d < D; ++d) yp[d] = y0[d];
                    typename PX::Cache c;
                    PX::prepare_flags(q, yp, c, tr, pass ? br1 : br0, pass ? nr1 : nr0);
                    St::explicit_from(q, rot, yp, c, B, w, dt);
#pragma unroll
                    for (int d = 0; d < D; ++d) y[d] = pass ? F2(lane0(y[d]), lane1(yp[d])) : yp[d];
                }
                F2 o[OUT];
                PX::out_t(y, o, tr);
                acc.add(o);
                if (++wpos == W32) {  // window end: uniform across the CTA
                    wpos = 0;
                    const unsigned long long kw = (g + 1) / W;
                    const int slot = static_cast<int>(kw - s0 / W - 1);
                    double* const traj = e.traj;
                    const int lane_id = threadIdx.x & 31;
#pragma unroll
                    for (int k = 0; k < 2; ++k) {
                        const double mom = active[k] ? e.moment[p[k]] : 0.0;
                        double* const partial = e.partial + ((p[k] >> 5) * e.slots + slot) * OUT;
                        const bool rec = traj && active[k] && (p[k] + 1) % e.traj_stride == 0;
                        const unsigned long long ti = rec ? (p[k] + 1) / e.traj_stride - 1 : 0;
                        double mine = 0.0;
#pragma unroll
                        for (int c = 0; c < OUT; ++c) {
                            const float v = active[k] ? lane(acc.get_sum(c), k) / static_cast<float>(static_cast<double>(W)) : 0.0f;
                            const double vd = static_cast<double>(v);
                            if (rec) traj[(kw * OUT + c) * e.traj_n + ti] = vd;
                            const double ws = warp_sum(active[k] ? weight_of<PROB>(c, mom) * vd : 0.0);
                            if (lane_id == c) mine = ws;
                        }
                        if (lane_id < OUT) partial[lane_id] = mine;
                    }
#pragma unroll
                    for (int c = 0; c < OUT; ++c) acc.clear_sum(c);
                }
            }
        }
#pragma unroll
        for (int k = 0; k < 2; ++k) {
            if (!active[k]) continue;
            float* st = static_cast<float*>(e.state);
            float* ksw = static_cast<float*>(e.ksum);
            float* kcw = static_cast<float*>(e.kcomp);
            bool finite = true;
#pragma unroll
            for (int i = 0; i < D; ++i) {
                const float v = lane(y[i], k);
                st[i * Np + p[k]] = v;
                finite = finite && isfinite(v);
            }
#pragma unroll
            for (int c = 0; c < OUT; ++c) {
                ksw[c * Np + p[k]] = lane(acc.get_sum(c), k);
                kcw[c * Np + p[k]] = lane(acc.get_comp(c), k);
            }
            if (!finite) e.status[p[k]] = 1;
        }
    }
}

}  // namespace sp
