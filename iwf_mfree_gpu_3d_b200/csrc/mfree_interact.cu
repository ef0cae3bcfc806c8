// mfree_interact.cu -- the pair loop and the fused per-particle rest of the step.
//
// Reference path replaced (src/leap_frog.cu:153-171):
//   do_interactions_monaghan  interactions_gpu.cu:152-471 (CSPM pre-pass, velocity
//                             gradient, stress divergence with artificial stress,
//                             artificial viscosity, XSPH, Brookshaw conduction)
//   do_interactions_heat      interactions_gpu.cu:89-150 (PSE conduction)
//   do_material_stress_rate_jaumann, do_contmech_continuity/momentum/advection
//                             actions_gpu.cu:134-300
//   correct                   leap_frog.cu:72-100
//   do_plasticity_johnson_cook actions_gpu.cu:371-449
//   do_reset_contact_forces, do_boundary_conditions(_thermal), do_move_tool_particles
//                             leap_frog.cu:102-119, actions_gpu.cu:55-68,451-487
//                             (particles inside a tool box defer these to k_finalize)
//
// Work decomposition: a warp owns 32 consecutive sorted particles.  It walks
// them in LPP rounds; in each round every group of LPP lanes serves one
// particle.  The 5x5x5 cell stencil is read as 25 contiguous particle ranges
// (five consecutive z cells of one (x, y) column are consecutive in the sorted
// order).  Pass A streams all candidates through the lanes: it tests the
// support, accumulates PSE (which sums every stencil candidate) and the CSPM
// matrix, and compacts the in-support neighbours into a shared-memory queue
// with a ballot.  Pass B runs the full pair body on the queue only -- the
// reference evaluates every candidate, ~3.5x more work, and candidates outside
// the support contribute exact zeros there.  Accumulators are reduced across
// the group with xor shuffles; after the LPP rounds each lane runs the
// per-particle epilogue for one particle.
#include "mfree_kernels.cuh"

namespace mfree {

template <int LPP> struct WarpSmem {
    static constexpr int G = 32 / LPP;
    int cbase[G][25];
    int cpref[G][26];
    int q[G][QCAP];
    float res[32][NRES + 1];
};

// 2x2 minors of the column-major (GLM) 3x3 in m[c*3+r]
__device__ __forceinline__ float det3(const float *m) {
    auto A = [&](int r, int c) { return m[c * 3 + r]; };
    return A(0, 0) * (A(1, 1) * A(2, 2) - A(1, 2) * A(2, 1)) - A(1, 0) * (A(0, 1) * A(2, 2) - A(0, 2) * A(2, 1)) +
           A(2, 0) * (A(0, 1) * A(1, 2) - A(0, 2) * A(1, 1));
}
__device__ __forceinline__ void inv3(const float *m, float det, float *o) {
    auto A = [&](int r, int c) { return m[c * 3 + r]; };
    const float id = 1.0f / det;
#pragma unroll
    for (int r = 0; r < 3; r++)
#pragma unroll
        for (int c = 0; c < 3; c++) {
            // o(r,c) = cofactor(c,r)/det
            const int r0 = (c + 1) % 3, r1 = (c + 2) % 3, c0 = (r + 1) % 3, c1 = (r + 2) % 3;
            o[c * 3 + r] = (A(r0, c0) * A(r1, c1) - A(r0, c1) * A(r1, c0)) * id;
        }
}

struct IData {
    float x, y, z, vx, vy, vz, rho, c, h, T, tool;
    float h1, fac;
    float s[6];  // sigma_i xx yy zz xy xz yz
    float R[6];  // R_i
};

// gradient factor of cubic_spline (kernels.cuh:26-69): value w and
// dfac = der*fac with grad W = dfac * (x_i - x_j)
__device__ __forceinline__ void spline(float r2, float h1, float fac, float &w, float &dfac) {
    const float rinv = rsqrtf(r2);
    const float r = r2 * rinv;
    const float q = r * h1;
    float val, der;
    if (q > 1.f) {
        const float t = 2.f - q, t2 = t * t;
        val = 0.25f * t2 * t;
        der = -0.75f * t2 * h1 * rinv;
    } else {
        val = 1.f - 1.5f * q * q * (1.f - 0.5f * q);
        der = -3.0f * q * (1.f - 0.75f * q) * h1 * rinv;
    }
    w = val * fac;
    dfac = der * fac;
}

template <bool CSPM, int COND>
__device__ __forceinline__ void pair_body(const Params &P, const IData &I, const float *invB, const float4 Pj,
                                          const float4 Vj, const float4 Aj, const float4 Bj, const float4 Rj,
                                          const float4 Cj, float *acc) {
    const float dx = I.x - Pj.x, dy = I.y - Pj.y, dz = I.z - Pj.z;
    const float r2 = dist2_rn(dx, dy, dz);
    float w, dfac;
    spline(r2, I.h1, I.fac, w, dfac);
    float gx = dfac * dx, gy = dfac * dy, gz = dfac * dz;
    if (CSPM) {
        const float ux = gx * invB[0] + gy * invB[3] + gz * invB[6];
        const float uy = gx * invB[1] + gy * invB[4] + gz * invB[7];
        const float uz = gx * invB[2] + gy * invB[5] + gz * invB[8];
        gx = ux; gy = uy; gz = uz;
    }
    const bool mech = !(I.tool == 1.f) && !(Pj.w == 1.f);
    const float volj = Cj.w;
    if (mech) {
        const float dvx = Vj.x - I.vx, dvy = Vj.y - I.vy, dvz = Vj.z - I.vz;
        const float ax = dvx * volj, ay = dvy * volj, az = dvz * volj;
        acc[0] = fmaf(ax, gx, acc[0]); acc[1] = fmaf(ax, gy, acc[1]); acc[2] = fmaf(ax, gz, acc[2]);
        acc[3] = fmaf(ay, gx, acc[3]); acc[4] = fmaf(ay, gy, acc[4]); acc[5] = fmaf(ay, gz, acc[5]);
        acc[6] = fmaf(az, gx, acc[6]); acc[7] = fmaf(az, gy, acc[7]); acc[8] = fmaf(az, gz, acc[8]);
        float Rxx = 0.f, Ryy = 0.f, Rzz = 0.f, Rxy = 0.f, Rxz = 0.f, Ryz = 0.f;
        if (P.wdeltap > 0.f) {
            float fab = w / P.wdeltap;
            fab *= fab;
            fab *= fab;
            Rxx = fab * (I.R[0] + Rj.x);
            Ryy = fab * (I.R[1] + Rj.y);
            Rzz = fab * (I.R[2] + Rj.z);
            Rxy = fab * (I.R[3] + Rj.w);
            Rxz = fab * (I.R[4] + Cj.x);
            Ryz = fab * (I.R[5] + Cj.y);
        }
        const float txx = I.s[0] + Aj.x + Rxx, tyy = I.s[1] + Aj.y + Ryy, tzz = I.s[2] + Aj.z + Rzz;
        const float txy = I.s[3] + Aj.w + Rxy, txz = I.s[4] + Bj.x + Rxz, tyz = I.s[5] + Bj.y + Ryz;
        acc[9] = fmaf(txx, gx, fmaf(txy, gy, fmaf(txz, gz, acc[9])));
        acc[10] = fmaf(txy, gx, fmaf(tyy, gy, fmaf(tyz, gz, acc[10])));
        acc[11] = fmaf(txz, gx, fmaf(tyz, gy, fmaf(tzz, gz, acc[11])));
        const float vr = -(dvx * dx + dvy * dy + dvz * dz);  // (v_i - v_j).(x_i - x_j)
        const float rhoij = 0.5f * (I.rho + Vj.w);
        const float irho = 1.0f / rhoij;
        if (vr < 0.f) {
            const float cij = 0.5f * (I.c + Bj.z), hij = 0.5f * (I.h + Bj.w);
            const float mu = (hij * vr) / (r2 + P.av_eta * P.av_eta * hij * hij);
            const float pij = (-P.av_alpha * cij * mu + P.av_beta * mu * mu) * irho;
            acc[12] = fmaf(-pij, gx, acc[12]);
            acc[13] = fmaf(-pij, gy, acc[13]);
            acc[14] = fmaf(-pij, gz, acc[14]);
        }
        const float xw = w * irho;
        acc[15] = fmaf(-xw, dvx, acc[15]);  // (w/rho_ij)(v_i - v_j)
        acc[16] = fmaf(-xw, dvy, acc[16]);
        acc[17] = fmaf(-xw, dvz, acc[17]);
    }
    if (COND == MFREE_COND_BROOKSHAW) {
        // 2 (m/rho_j)(T_i - T_j) e.grad W / r = 2 V_j (T_i - T_j) (d.grad W)/r^2; factor 2 in the epilogue
        acc[18] = fmaf(volj * (I.T - Cj.z), (dx * gx + dy * gy + dz * gz) / r2, acc[18]);
    }
}

// ------------------------------------------------------------ epilogue --
template <bool PREC, int COND>
__device__ void epilogue(const StepArgs &a, int i, const float *res) {
    const Params &P = a.p;
    const State &S = a.b;
    float4 pos = S.pos4[i], vel = S.vel4[i], sa = S.sa4[i], sb = S.sb4[i];
    float4 da = S.da4[i], dv = S.dv4[i], dsa = S.dsa4[i], dsb = S.dsb4[i];
    float4 ft = S.ft4[i], fc = S.fc4[i];
    float4 lo = make_float4(0.f, 0.f, 0.f, 0.f), lob = lo;
    if (PREC) {
        lo = S.lo4[i];
        lob = S.lo4b[i];
    }
    const float dt = P.dt;
    const HalfStep hs = half_step<PREC>(0.5f * dt, pos, vel, sa, sb, da, dv, dsa, dsb, lo, lob);
    const float tool_p = fc.w;
    const bool tool = tool_p == 1.f;
    const float fixed = dsb.w;
    // ---- rates
    float pt[3], vt[3], St[6], rho_t, T_t;
    if (!tool) {
        float L[9];
#pragma unroll
        for (int k = 0; k < 9; k++) L[k] = res[k];
        jaumann(L, hs.S, P.G, St);
        rho_t = -hs.rho * (L[0] + L[4] + L[8]);
        const float im = 1.0f / P.mass;
        vt[0] = P.mass * (res[12] + res[9]) + fc.x * im + ft.x * im;
        vt[1] = P.mass * (res[13] + res[10]) + fc.y * im + ft.y * im;
        vt[2] = P.mass * (res[14] + res[11]) + fc.z * im + ft.z * im;
        const float xf = -P.xspheps * P.mass;
        pt[0] = fmaf(xf, res[15], hs.vx);
        pt[1] = fmaf(xf, res[16], hs.vy);
        pt[2] = fmaf(xf, res[17], hs.vz);
    } else {
        pt[0] = pt[1] = pt[2] = 0.f;
        vt[0] = vt[1] = vt[2] = 0.f;
        St[0] = dsa.x; St[1] = dsa.y; St[2] = dsa.z; St[3] = dsa.w; St[4] = dsb.x; St[5] = dsb.y;
        rho_t = da.w;
    }
    T_t = dv.w;
    if (COND == MFREE_COND_BROOKSHAW) {
        const float al = tool_p == 0.f ? P.wp_alpha : P.tool_alpha;
        if (al != 0.f) T_t = al * (2.0f * res[18]);
    } else if (COND == MFREE_COND_PSE) {
        if (P.wp_alpha != 0.f) {
            const float al = tool ? P.tool_alpha : P.wp_alpha;
            const float h = pos.w, h2 = h * h;
            const float coef = 4.0f / (h2 * h2 * h * 5.5683279968317078f);  // pi^1.5
            T_t = al * coef * res[18];
        }
    }
    // ---- corrector x1 = x0 + dt * xdot (leap_frog.cu:72-100)
    if (PREC) {
        acc_comp(pos.x, lo.x, dt, pt[0]);
        acc_comp(pos.y, lo.y, dt, pt[1]);
        acc_comp(pos.z, lo.z, dt, pt[2]);
        acc_comp(vel.x, lo.w, dt, vt[0]);
        acc_comp(vel.y, lob.x, dt, vt[1]);
        acc_comp(vel.z, lob.y, dt, vt[2]);
    } else {
        pos.x = fmaf(dt, pt[0], pos.x);
        pos.y = fmaf(dt, pt[1], pos.y);
        pos.z = fmaf(dt, pt[2], pos.z);
        vel.x = fmaf(dt, vt[0], vel.x);
        vel.y = fmaf(dt, vt[1], vel.y);
        vel.z = fmaf(dt, vt[2], vel.z);
    }
    float s[6] = {fmaf(dt, St[0], sa.x), fmaf(dt, St[1], sa.y), fmaf(dt, St[2], sa.z),
                  fmaf(dt, St[3], sa.w), fmaf(dt, St[4], sb.x), fmaf(dt, St[5], sb.y)};
    vel.w = fmaf(dt, rho_t, vel.w);  // rho
    float T = fmaf(dt, T_t, sb.z);
    float eps = sb.w, epsd = dsb.z;
    // ---- Johnson-Cook radial return (actions_gpu.cu:371-449)
    if (P.plastic && !tool) {
        const float nS = sqrtf(s[0] * s[0] + s[1] * s[1] + s[2] * s[2] + 2.f * (s[3] * s[3] + s[5] * s[5] + s[4] * s[4]));
        float Tc = T;
        if (P.jc_clamp != 0.f) Tc = Tc > P.jc_Tmelt ? P.jc_Tmelt - 1.f : Tc;
        const float svm = 1.22474487139158905f * nS;
        const float sY = jc_sigma_yield(P, eps, epsd, Tc);
        if (svm < sY) {
            epsd = 0.f;
        } else {
            bool failed = false;
            const float s23 = 0.81649658092772603f;
            const float init = fmaxf(epsd * dt * s23, 1e-8f);
            const float dl = jc_secant(P, init, nS, eps, Tc, dt, failed);
            if (failed) atomicAdd(&a.clk->secant_failures, 1ull);
            const float e1 = eps + s23 * fmaxf(dl, 0.f);
            const float ed1 = s23 * fmaxf(dl, 0.f) / dt;
            const float f = dl * 2.f * P.G / nS;
#pragma unroll
            for (int k = 0; k < 6; k++) s[k] = s[k] - s[k] * f;
            if (P.wp_tq != 0.f) {
                const float sY2 = jc_sigma_yield(P, e1, ed1, Tc);
                T += P.wp_tq / (P.wp_cp * vel.w) * (e1 - eps) * sY2;
            }
            eps = e1;
            epsd = ed1;
        }
    }
    // ---- contact reset; particles inside a tool box finish in k_finalize
    const bool deferred = !tool && contact_candidate(a, pos.x, pos.y, pos.z);
    fc.x = fc.y = fc.z = 0.f;  // w keeps tool_p
    ft.x = ft.y = ft.z = 0.f;  // w keeps blanked
    if (!deferred) {
        if (!tool && fixed != 0.f) {
            const float4 bc = S.bc4[i];
            vel.x = bc.x; vel.y = bc.y; vel.z = bc.z;
            if (PREC) { lo.w = 0.f; lob.x = lob.y = 0.f; }
            pt[0] = pt[1] = pt[2] = 0.f;
            vt[0] = vt[1] = vt[2] = 0.f;
        }
        if (P.thermal && fixed == 1.f) T = P.wp_Tinit;
        if (P.diagnostics) a.s.nrm[i] = make_float4(0.f, 0.f, 0.f, 0.f);
    }
    if (tool) {  // do_move_tool_particles
        if (PREC) {
            acc_comp(pos.x, lo.x, dt, P.tool0_vel[0]);
            acc_comp(pos.y, lo.y, dt, P.tool0_vel[1]);
            acc_comp(pos.z, lo.z, dt, P.tool0_vel[2]);
        } else {
            pos.x = fmaf(P.tool0_vel[0], dt, pos.x);
            pos.y = fmaf(P.tool0_vel[1], dt, pos.y);
            pos.z = fmaf(P.tool0_vel[2], dt, pos.z);
        }
    }
    S.pos4[i] = pos;
    S.vel4[i] = vel;
    S.sa4[i] = make_float4(s[0], s[1], s[2], s[3]);
    S.sb4[i] = make_float4(s[4], s[5], T, eps);
    S.da4[i] = make_float4(pt[0], pt[1], pt[2], rho_t);
    S.dv4[i] = make_float4(vt[0], vt[1], vt[2], T_t);
    S.dsa4[i] = make_float4(St[0], St[1], St[2], St[3]);
    S.dsb4[i] = make_float4(St[4], St[5], epsd, fixed);
    S.fc4[i] = fc;
    S.ft4[i] = ft;
    if (PREC) {
        S.lo4[i] = lo;
        S.lo4b[i] = lob;
    }
    if (P.diagnostics) a.s.nnb[i] = __float_as_int(res[19]);
}

// ---------------------------------------------------------- pair kernel --
template <int LPP, bool CSPM, int COND, bool PREC>
__global__ void __launch_bounds__(INTERACT_WARPS * 32) k_interact(StepArgs a) {
    constexpr int G = 32 / LPP;
    __shared__ WarpSmem<LPP> smem[INTERACT_WARPS];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / LPP, sl = lane - g * LPP;
    WarpSmem<LPP> &sm = smem[warp];
    const Params &P = a.p;
    const int N = a.clk->n_active;
    const int nbatch = (N + 31) >> 5;
    const unsigned lt_mask = (1u << lane) - 1u;
    const unsigned gmask = LPP == 32 ? 0xffffffffu : (((1u << LPP) - 1u) << (g * LPP));
    const int nx = P.gnx, ny = P.gny, nz = P.gnz;
    const float4 *__restrict__ RP = a.r.P;
    const float4 *__restrict__ RV = a.r.V;
    const float4 *__restrict__ RA = a.r.A;
    const float4 *__restrict__ RB = a.r.B;
    const float4 *__restrict__ RR = a.r.R;
    const float4 *__restrict__ RC = a.r.C;
    const int *__restrict__ first = a.s.first;

    for (int batch = blockIdx.x * INTERACT_WARPS + warp; batch < nbatch; batch += gridDim.x * INTERACT_WARPS) {
        const int base = batch << 5;
#pragma unroll 1
        for (int rnd = 0; rnd < LPP; rnd++) {
            const int i = base + rnd * G + g;
            const bool valid = i < N;
            const int ii = valid ? i : base;
            IData I;
            {
                const float4 Pi = RP[ii], Vi = RV[ii], Ai = RA[ii], Bi = RB[ii], Ri = RR[ii], Ci = RC[ii];
                I.x = Pi.x; I.y = Pi.y; I.z = Pi.z; I.tool = Pi.w;
                I.vx = Vi.x; I.vy = Vi.y; I.vz = Vi.z; I.rho = Vi.w;
                I.s[0] = Ai.x; I.s[1] = Ai.y; I.s[2] = Ai.z; I.s[3] = Ai.w; I.s[4] = Bi.x; I.s[5] = Bi.y;
                I.c = Bi.z; I.h = Bi.w;
                I.R[0] = Ri.x; I.R[1] = Ri.y; I.R[2] = Ri.z; I.R[3] = Ri.w; I.R[4] = Ci.x; I.R[5] = Ci.y;
                I.T = Ci.z;
                I.h1 = 1.0f / I.h;
                I.fac = 0.31830988618379067f * I.h1 * I.h1 * I.h1;
            }
            // the 25 (x, y) columns of the 5x5x5 stencil around the particle's cell
            {
                const unsigned key = a.s.key_sorted[ii];
                const int nyz = ny * nz;
                const int gi = int(key) / nyz, rem = int(key) - gi * nyz, gj = rem / nz, gk = rem - gj * nz;
                const int z0 = max(gk - 2, 0), z1 = min(gk + 2, nz - 1);
                for (int c = sl; c < 25; c += LPP) {
                    const int cx = gi + c / 5 - 2, cy = gj + c % 5 - 2;
                    int s = 0, e = 0;
                    if (valid && cx >= 0 && cx < nx && cy >= 0 && cy < ny) {
                        const int cb = (cx * ny + cy) * nz;
                        s = first[cb + z0];
                        e = first[cb + z1 + 1];
                    }
                    sm.cbase[g][c] = s;
                    sm.cpref[g][c] = e - s;
                }
            }
            __syncwarp();
            if (sl == 0) {
                int acc = 0;
                for (int c = 0; c < 25; c++) {
                    const int l = sm.cpref[g][c];
                    sm.cpref[g][c] = acc;
                    acc += l;
                }
                sm.cpref[g][25] = acc;
            }
            __syncwarp();
            const int total = sm.cpref[g][25];
            int maxtotal = total;
#pragma unroll
            for (int o = 16; o >= LPP; o >>= 1) maxtotal = max(maxtotal, __shfl_xor_sync(0xffffffffu, maxtotal, o));

            // ---- pass A: support test, PSE, CSPM matrix, queue
            const float inv_h2 = I.h1 * I.h1;
            int col = 0, qn = 0, cnt = 0;
            float pse = 0.f;
            float Bm[9];
#pragma unroll
            for (int k = 0; k < 9; k++) Bm[k] = 0.f;
            for (int k0 = 0; k0 < maxtotal; k0 += LPP) {
                const int k = k0 + sl;
                bool ins = false;
                int j = 0;
                if (k < total) {
                    while (sm.cpref[g][col + 1] <= k) col++;
                    j = sm.cbase[g][col] + (k - sm.cpref[g][col]);
                    const float4 Pj = RP[j];
                    const float dx = I.x - Pj.x, dy = I.y - Pj.y, dz = I.z - Pj.z;
                    const float r2 = dist2_rn(dx, dy, dz);
                    ins = in_support(r2, I.h);
                    if (COND == MFREE_COND_PSE || CSPM) {
                        const float4 Cj = RC[j];
                        if (COND == MFREE_COND_PSE) pse = fmaf((Cj.z - I.T) * Cj.w, __expf(-r2 * inv_h2), pse);
                        if (CSPM && ins && !(I.tool == 1.f) && !(Pj.w == 1.f)) {
                            float w, dfac;
                            spline(r2, I.h1, I.fac, w, dfac);
                            const float d[3] = {dx, dy, dz};
                            const float gr[3] = {dfac * dx, dfac * dy, dfac * dz};
#pragma unroll
                            for (int c = 0; c < 3; c++)
#pragma unroll
                                for (int r = 0; r < 3; r++) Bm[c * 3 + r] = fmaf(-Cj.w * d[r], gr[c], Bm[c * 3 + r]);
                        }
                    }
                }
                cnt += ins ? 1 : 0;
                const unsigned m = __ballot_sync(0xffffffffu, ins) & gmask;
                if (ins) {
                    const int pos = qn + __popc(m & lt_mask);
                    if (pos < QCAP) sm.q[g][pos] = j;
                }
                qn += __popc(m);
            }
            __syncwarp();
            float invB[9] = {1.f, 0.f, 0.f, 0.f, 1.f, 0.f, 0.f, 0.f, 1.f};
            if (CSPM) {
#pragma unroll
                for (int o = LPP / 2; o >= 1; o >>= 1)
#pragma unroll
                    for (int k = 0; k < 9; k++) Bm[k] += __shfl_xor_sync(0xffffffffu, Bm[k], o);
                const float det = det3(Bm);
                if (det > 9.99999994e-9f) inv3(Bm, det, invB);
            }
            // ---- pass B: pair body on the in-support queue
            float acc[19];
#pragma unroll
            for (int k = 0; k < 19; k++) acc[k] = 0.f;
            const int qv = min(qn, QCAP);
            int maxq = qv;
#pragma unroll
            for (int o = 16; o >= LPP; o >>= 1) maxq = max(maxq, __shfl_xor_sync(0xffffffffu, maxq, o));
            for (int q0 = 0; q0 < maxq; q0 += LPP) {
                const int q = q0 + sl;
                if (q < qv) {
                    const int j = sm.q[g][q];
                    pair_body<CSPM, COND>(P, I, invB, RP[j], RV[j], RA[j], RB[j], RR[j], RC[j], acc);
                }
            }
            // more in-support neighbours than the queue holds: rescan, take the rest
            if (__any_sync(0xffffffffu, qn > QCAP)) {
                int col2 = 0, ord = 0;
                for (int k0 = 0; k0 < maxtotal; k0 += LPP) {
                    const int k = k0 + sl;
                    bool ins = false;
                    int j = 0;
                    if (k < total && qn > QCAP) {
                        while (sm.cpref[g][col2 + 1] <= k) col2++;
                        j = sm.cbase[g][col2] + (k - sm.cpref[g][col2]);
                        const float4 Pj = RP[j];
                        ins = in_support(dist2_rn(I.x - Pj.x, I.y - Pj.y, I.z - Pj.z), I.h);
                    }
                    const unsigned m = __ballot_sync(0xffffffffu, ins) & gmask;
                    const int pos = ord + __popc(m & lt_mask);
                    if (ins && pos >= QCAP)
                        pair_body<CSPM, COND>(P, I, invB, RP[j], RV[j], RA[j], RB[j], RR[j], RC[j], acc);
                    ord += __popc(m);
                }
            }
            if (COND == MFREE_COND_PSE) acc[18] = pse;
            // ---- reduce over the group's lanes
#pragma unroll
            for (int o = LPP / 2; o >= 1; o >>= 1) {
#pragma unroll
                for (int k = 0; k < 19; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
                cnt += __shfl_xor_sync(0xffffffffu, cnt, o);
            }
            if (sl == 0) {
                float *rs = sm.res[rnd * G + g];
#pragma unroll
                for (int k = 0; k < 19; k++) rs[k] = acc[k];
                rs[19] = __int_as_float(cnt);
            }
            __syncwarp();
        }
        const int i = base + lane;
        if (i < N) epilogue<PREC, COND>(a, i, sm.res[lane]);
        __syncwarp();
    }
}

// ------------------------------------------------------------ dispatch --
template <int LPP, bool CSPM, int COND, bool PREC>
static cudaError_t launch_one(const StepArgs &a, int grid, cudaStream_t s) {
    k_interact<LPP, CSPM, COND, PREC><<<grid, INTERACT_WARPS * 32, 0, s>>>(a);
    return cudaGetLastError();
}

template <int LPP>
static cudaError_t launch_lpp(const StepArgs &a, int grid, cudaStream_t s) {
    const bool cspm = a.p.cspm != 0, prec = a.p.precision != 0;
    const int cond = a.p.conduction;
#define MFREE_CASE(C, CO, PR) \
    if (cspm == C && cond == CO && prec == PR) return launch_one<LPP, C, CO, PR>(a, grid, s);
    MFREE_CASE(false, MFREE_COND_NONE, false)
    MFREE_CASE(false, MFREE_COND_BROOKSHAW, false)
    MFREE_CASE(false, MFREE_COND_PSE, false)
    MFREE_CASE(true, MFREE_COND_NONE, false)
    MFREE_CASE(true, MFREE_COND_BROOKSHAW, false)
    MFREE_CASE(true, MFREE_COND_PSE, false)
    MFREE_CASE(false, MFREE_COND_NONE, true)
    MFREE_CASE(false, MFREE_COND_BROOKSHAW, true)
    MFREE_CASE(false, MFREE_COND_PSE, true)
    MFREE_CASE(true, MFREE_COND_NONE, true)
    MFREE_CASE(true, MFREE_COND_BROOKSHAW, true)
    MFREE_CASE(true, MFREE_COND_PSE, true)
#undef MFREE_CASE
    return cudaErrorInvalidValue;
}

cudaError_t launch_interact(const StepArgs &a, int lpp, int grid, cudaStream_t s) {
    switch (lpp) {
        case 4: return launch_lpp<4>(a, grid, s);
        case 8: return launch_lpp<8>(a, grid, s);
        case 16: return launch_lpp<16>(a, grid, s);
        case 32: return launch_lpp<32>(a, grid, s);
        default: return cudaErrorInvalidValue;
    }
}

// persistent-style grid: enough blocks to fill every SM several times over,
// never more than there are 32-particle batches
int interact_grid_size(int lpp, int n_init, int num_sms) {
    (void)lpp;
    const int batches = (n_init + 31) / 32;
    const int blocks_needed = (batches + INTERACT_WARPS - 1) / INTERACT_WARPS;
    const int cap = num_sms * 16;
    return blocks_needed < cap ? (blocks_needed > 0 ? blocks_needed : 1) : cap;
}

}  // namespace mfree
