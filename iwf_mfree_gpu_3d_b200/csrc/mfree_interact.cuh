// mfree_interact.cuh -- the pair loop and the fused per-particle rest of the step
// (kernel templates; mfree_interact.cu instantiates and launches them).
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
//                             (particles inside a tool box defer these to kb_finalize)
//
// Work decomposition: a persistent block (640 threads, one per SM) pulls
// tiles of 4 x 4 x D cells (D = Params::tile_z, 6 by default) of every scene
// of the table from one work counter.  The tile's particles are 16 contiguous
// ranges of the sorted order; the records their 5x5x5 stencils touch are the
// 64 contiguous column ranges of the 8 x 8 x (D+4)-cell halo, staged into
// shared memory with two bulk copies per column, its P records and the
// interleaved rest (TMA cp.async.bulk, completion counted on an mbarrier,
// bounded waits).  Each
// target is served by a group of LPP lanes.  Pass A streams the target's
// candidates (25 column ranges of the staged halo) through the lanes: support
// test, PSE (which sums every stencil candidate) and a ballot that compacts
// the in-support neighbours into a queue.  The CSPM pass (symmetric matrix)
// and the pair pass run on the queue only -- the reference evaluates the pair
// body for every candidate, ~3.5x more work, and candidates outside the
// support contribute exact zeros there.  Accumulators are reduced across the
// group with xor shuffles; then one thread per target runs the per-particle
// epilogue.  The epilogue needs at most TCAP = 320 threads; during the
// epilogue of a tile's last pass the other 320 already prepare the next tile
// (its target ranges, halo table and staging copies), so those copies land
// while the epilogue runs.
#pragma once

#include "mfree_kernels.cuh"

namespace mfree {

// The CSPM matrix B = sum V_j (x_i - x_j) (x) grad W_ij is symmetric (grad W
// is parallel to x_i - x_j), and so is its inverse: both are kept as the six
// entries xx, yy, zz, xy, xz, yz.
__device__ __forceinline__ float det3s(const float *m) {
    return m[0] * (m[1] * m[2] - m[5] * m[5]) - m[3] * (m[3] * m[2] - m[4] * m[5]) + m[4] * (m[3] * m[5] - m[4] * m[1]);
}
// inverse by cofactors (cofactor(r, c) / det; symmetric)
__device__ __forceinline__ void inv3s(const float *m, float det, float *o) {
    const float id = 1.0f / det;
    o[0] = (m[1] * m[2] - m[5] * m[5]) * id;  // xx
    o[1] = (m[0] * m[2] - m[4] * m[4]) * id;  // yy
    o[2] = (m[0] * m[1] - m[3] * m[3]) * id;  // zz
    o[3] = (m[4] * m[5] - m[3] * m[2]) * id;  // xy
    o[4] = (m[3] * m[5] - m[4] * m[1]) * id;  // xz
    o[5] = (m[3] * m[4] - m[0] * m[5]) * id;  // yz
}

// the target's terms of the pair loop; its own sigma and R enter the stress
// divergence only through the group's sums (see pair_body) and are read after
// the loop
struct IData {
    float x, y, z, vx, vy, vz, rho, c, h, T, tool;
    float h1, fac;
};

// gradient factor of cubic_spline (kernels.cuh:26-69): value w and
// dfac = der*fac with grad W = dfac * (x_i - x_j)
__device__ __forceinline__ void spline(float r2, float h1, float fac, float &w, float &dfac) {
    float rinv;  // r2 >= 1e-8 here: never a denormal
    asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(rinv) : "f"(r2));
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

// the scene constants of the pair body, held in registers for a target's
// pair loop (read from the shared-memory arguments in the loop they were
// loaded again for every pair: 1.869 -> 1.847 ms on the 1M step)
struct PairConst {
    float inv_wdeltap, eta2, alpha, beta;  // 1 / wdeltap, eta^2 (as eta * eta), AV alpha and beta
    bool art;                              // artificial stress on (wdeltap > 0)
};
template <bool CSPM, int COND>
__device__ __forceinline__ void pair_body(const PairConst &P, const IData &I, const float *invB, const float4 Pj,
                                          const float4 Vj, const float4 Aj, const float4 Bj, const float4 Rj,
                                          const float4 Cj, float *acc) {
    const float dx = I.x - Pj.x, dy = I.y - Pj.y, dz = I.z - Pj.z;
    const float r2 = dist2_rn(dx, dy, dz);
    float w, dfac;
    spline(r2, I.h1, I.fac, w, dfac);
    float gx = dfac * dx, gy = dfac * dy, gz = dfac * dz;
    if (CSPM) {
        const float ux = gx * invB[0] + gy * invB[3] + gz * invB[4];
        const float uy = gx * invB[3] + gy * invB[1] + gz * invB[5];
        const float uz = gx * invB[4] + gy * invB[5] + gz * invB[2];
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
        // sum_j (sigma_i + sigma_j + fab (R_i + R_j)) g
        //   = sum_j (sigma_j + fab R_j) g + sigma_i sum_j g + R_i sum_j fab g:
        // slots 19-21 and 22-24 hold sum_j g and sum_j fab g, which the caller
        // multiplies by the target's sigma and R once
        float txx = Aj.x, tyy = Aj.y, tzz = Aj.z, txy = Aj.w, txz = Bj.x, tyz = Bj.y;
        if (P.art) {
            float fab = w * P.inv_wdeltap;
            fab *= fab;
            fab *= fab;
            txx = fmaf(fab, Rj.x, txx); tyy = fmaf(fab, Rj.y, tyy); tzz = fmaf(fab, Rj.z, tzz);
            txy = fmaf(fab, Rj.w, txy); txz = fmaf(fab, Cj.x, txz); tyz = fmaf(fab, Cj.y, tyz);
            acc[22] = fmaf(fab, gx, acc[22]); acc[23] = fmaf(fab, gy, acc[23]); acc[24] = fmaf(fab, gz, acc[24]);
        }
        acc[19] += gx; acc[20] += gy; acc[21] += gz;
        acc[9] = fmaf(txx, gx, fmaf(txy, gy, fmaf(txz, gz, acc[9])));
        acc[10] = fmaf(txy, gx, fmaf(tyy, gy, fmaf(tyz, gz, acc[10])));
        acc[11] = fmaf(txz, gx, fmaf(tyz, gy, fmaf(tzz, gz, acc[11])));
        const float vr = -(dvx * dx + dvy * dy + dvz * dz);  // (v_i - v_j).(x_i - x_j)
        const float rhoij = 0.5f * (I.rho + Vj.w);
        const float irho = __fdividef(1.0f, rhoij);
        {   // artificial viscosity for approaching pairs (vr < 0), without a branch
            const float cij = 0.5f * (I.c + Bj.z), hij = 0.5f * (I.h + Bj.w);
            const float mu = vr < 0.f ? __fdividef(hij * vr, r2 + P.eta2 * hij * hij) : 0.f;
            const float pij = (-P.alpha * cij * mu + P.beta * mu * mu) * irho;
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
        acc[18] = fmaf(volj * (I.T - Cj.z), __fdividef(dx * gx + dy * gy + dz * gz, r2), acc[18]);
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
        if (jc_clearly_elastic(P, svm, eps, epsd, Tc) || svm < 0.99f * jc_yield_stress_screen(P, eps, epsd, Tc) ||
            svm < jc_yield_stress(P, eps, epsd, Tc)) {
            epsd = 0.f;  // elastic
        } else {
            // FP64 secant from FP32 inputs, the result stored as float
            int failed = 0;
            const double init = fmax((double)(epsd * dt) * 0.81649658092772603, 1e-8);
            const float dl = (float)jc_secant(P, init, nS, eps, Tc, dt, &failed);
            if (failed) atomicAdd(&a.clk->secant_failures, 1ull);
            const float s23 = 0.81649658092772603f;  // sqrtf(2/3)
            const float e1 = eps + s23 * fmaxf(dl, 0.f);
            const float ed1 = s23 * fmaxf(dl, 0.f) / dt;
            // S - S / |S| * dl * 2 * G: the quotient and the product with dl in
            // float, the rest in double (the literal 2. promotes it)
#pragma unroll
            for (int k = 0; k < 6; k++) s[k] = (float)((double)s[k] - (double)(s[k] / nS * dl) * 2.0 * (double)P.G);
            if (P.wp_tq != 0.f) {
                const float sY2 = jc_yield_stress(P, e1, ed1, Tc);
                T += P.wp_tq / (P.wp_cp * vel.w) * (e1 - eps) * sY2;
            }
            eps = e1;
            epsd = ed1;
        }
    }
    // ---- contact reset; particles inside a tool box finish in kb_finalize
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
// Tile = TX x TY x TZ cells of the cell grid; its particles are 16 contiguous
// column ranges of the sorted order.  Their 5x5x5 stencils lie in the halo of
// HX x HY x HZ cells: 64 contiguous column ranges of the P records and of the
// interleaved rest, which two bulk copies per column (cp.async.bulk,
// completion counted on an mbarrier) stage into shared memory in the same
// layout.  A tile whose halo exceeds the staging capacity reads the same
// records from global memory instead.
constexpr int HX = TX + 4, HY = TY + 4;
constexpr int CSROW = TILE_Z_MAX + 5;  // cell starts kept per halo column
constexpr int NHC = HX * HY;           // halo columns
constexpr int NTC = TX * TY;           // target columns
// threads per block: 640 (20 warps, 96 registers a thread, a few spilled)
// beat 512 (16 warps, 128 registers) by about 2 % on the 1M-particle scene
// (CSPM + PSE) and by about 1 % on the mixed-size scenes (Brookshaw); 672 and
// more threads leave at most 80 registers a thread, and the spills win
template <bool CSPM> __host__ __device__ constexpr int tile_threads() { return 640; }
constexpr int TCAP = 320;              // targets per pass of a tile
constexpr int QCAP_T = 96;             // in-support queue per target before the rescan path

// The in-support queue and the column walk of a group.  A staged tile's
// record indices are below the staging capacity, so its queue entries are 16
// bits and a column-walk entry packs the column's end in the flattened order
// (low 16 bits) with the record-minus-flattened index offset (high 16 bits,
// signed): both lie within the capacity.  A tile read from global memory keeps
// 32-bit entries, placed in the staging area that such a tile leaves idle.
template <bool STAGED> struct Walk {
    using Q = unsigned short;
    using C = int;
    static __device__ __forceinline__ C pack(int end, int off) { return int(unsigned(off) << 16) | end; }
    static __device__ __forceinline__ int end(C w) { return w & 0xffff; }
    static __device__ __forceinline__ int off(C w) { return w >> 16; }
};
template <> struct Walk<false> {
    using Q = int;
    using C = int2;
    static __device__ __forceinline__ C pack(int end, int off) { return make_int2(end, off); }
    static __device__ __forceinline__ int end(C w) { return w.x; }
    static __device__ __forceinline__ int off(C w) { return w.y; }
};
constexpr int SMEM_LIMIT = 232448;     // per-block shared memory of sm_100
constexpr long long WAIT_CYCLES = 1ll << 30;  // bound of a staging wait (~0.5 s of SM clock)

template <int LPP, int TILE_WARPS> struct TileSmem {
    static constexpr int G = 32 / LPP;
    float res[TCAP][NRES + 1];
    int tgt[TCAP];       // sorted index of each target of the pass
    int tcell[TCAP];     // its cell: target column << 16 | z
    unsigned short q[TILE_WARPS][G][QCAP_T];
    // per stencil column of a group's target: end of its candidates in the
    // flattened order and record index minus flattened index (Walk<true>)
    int cwalk[TILE_WARPS][G][25];
    int cellstart[NHC][CSROW];
    int hoff[NHC];       // staged offset of a halo column
    int hstart[NHC];     // global start of a halo column
    int hlen[NHC];
    int tstart[NTC];
    int tpref[NTC + 1];
    unsigned long long bar;
    float4 org;        // stencil pruning of the current tile's scene: grid origin, 1 = on (no PSE only)
    int tile, total, staged, parity, scene;  // scene < 0: no tile left
    int next_args;     // scene whose arguments the second args buffer holds (-1: none)
    int ntile, nscene; // the prologue threads' candidate tile
    int2 pre_entry;    // tile-list entry fetched ahead for the next prologue
    int pre_ok;        // pre_entry is being fetched (cp.async)
    int list_n;        // entries of the tile list
};
__host__ __device__ constexpr size_t round128(size_t b) { return (b + 127) / 128 * 128; }
// shared memory: the tables, the scene's arguments, the staged records
template <int LPP, int W> __host__ __device__ constexpr size_t args_offset() {
    return round128(sizeof(TileSmem<LPP, W>));
}
template <int LPP, int W> __host__ __device__ constexpr size_t rec_offset() {
    return args_offset<LPP, W>() + 2 * round128(sizeof(StepArgs));  // the current and the next tile's scene
}
template <int LPP, int W> __host__ __device__ constexpr int rec_capacity() {
    return int((SMEM_LIMIT - rec_offset<LPP, W>()) / (REC_N * sizeof(float4)));
}

__device__ __forceinline__ unsigned smem_u32(const void *p) { return unsigned(__cvta_generic_to_shared(p)); }
__device__ __forceinline__ void mbar_init(unsigned long long *b, unsigned n) {
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(b)), "r"(n) : "memory");
}
__device__ __forceinline__ void mbar_expect(unsigned long long *b, unsigned bytes) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(b)), "r"(bytes) : "memory");
}
__device__ __forceinline__ bool mbar_try(unsigned long long *b, unsigned parity) {
    unsigned ok;
    asm volatile(
        "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
        : "=r"(ok)
        : "r"(smem_u32(b)), "r"(parity)
        : "memory");
    return ok != 0;
}
__device__ __forceinline__ void bulk_to_smem(void *dst, const void *src, unsigned bytes, unsigned long long *b) {
    asm volatile("cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];" ::"r"(
                     smem_u32(dst)),
                 "l"(src), "r"(bytes), "r"(smem_u32(b))
                 : "memory");
}
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// inclusive scan over the LPP lanes of a group
template <int LPP> __device__ __forceinline__ int group_scan(int v, int sl) {
#pragma unroll
    for (int o = 1; o < LPP; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, v, o, LPP);
        if (sl >= o) v += y;
    }
    return v;
}

// the records of one kind at a fixed stride: P alone, the other five
// interleaved per particle
template <int S> struct RecView {
    const float4 *__restrict__ p;
    __device__ __forceinline__ const float4 &operator[](int j) const { return p[j * S]; }
};

// one target: stencil ranges, pass A (support, PSE, queue), CSPM pass over
// the queue, pair pass over the queue, group reduction
template <int LPP, bool CSPM, int COND, bool STAGED, class SM>
__device__ __forceinline__ void process_target(const StepArgs &a, SM &sm, float4 *spare, const float4 *RF, int rstride,
                                               int i, bool valid, int tt, int warp, int g, int sl, int lane, int X0,
                                               int Y0, int zl) {
    const Params &P = a.p;
    const int nx = P.gnx, ny = P.gny, nz = P.gnz;
    const unsigned lt_mask = (1u << lane) - 1u;
    const unsigned gmask = LPP == 32 ? 0xffffffffu : (((1u << LPP) - 1u) << (g * LPP));
    // the records of rstride particles (shared memory or global): P at RF,
    // V, A, B, R, C interleaved from RF + rstride
    const float4 *X = RF + rstride;
    const RecView<1> rP{RF};
    const RecView<REC_X> rV{X + (REC_V - 1)}, rA{X + (REC_A - 1)}, rB{X + (REC_B - 1)}, rR{X + (REC_R - 1)},
        rC{X + (REC_C - 1)};
    // the target's cell (from the pass's target table); its own records come
    // from the staged halo (its cell column is one of the halo's) or from
    // global memory
    const int tcell = sm.tcell[valid ? tt : 0];
    const int gi = X0 + (tcell >> 16) / TY, gj = Y0 + (tcell >> 16) % TY, gk = tcell & 0xffff;
    IData I;
    int si = i;  // the target's own record
    if (STAGED) {
        const int lc = (gi - X0 + 2) * HY + (gj - Y0 + 2);
        si = sm.hoff[lc] + (i - sm.hstart[lc]);
        if (!bounds_ok(a.clk, si, rstride)) si = 0;
    }
    {
        const float4 Pi = rP[si], Vi = rV[si], Bi = rB[si], Ci = rC[si];
        I.x = Pi.x; I.y = Pi.y; I.z = Pi.z; I.tool = Pi.w;
        I.vx = Vi.x; I.vy = Vi.y; I.vz = Vi.z; I.rho = Vi.w;
        I.c = Bi.z; I.h = Bi.w;
        I.T = Ci.z;
        I.h1 = 1.0f / I.h;
        I.fac = 0.31830988618379067f * I.h1 * I.h1 * I.h1;
    }
    using WK = Walk<STAGED>;
    typename WK::C *cw;
    typename WK::Q *qq;
    if (STAGED) {
        cw = reinterpret_cast<typename WK::C *>(sm.cwalk[warp][g]);
        qq = reinterpret_cast<typename WK::Q *>(sm.q[warp][g]);
    } else {  // 32-bit entries in the idle staging area
        constexpr int NG = int(sizeof(sm.q) / sizeof(sm.q[0][0]));  // groups of the block
        int *q32 = reinterpret_cast<int *>(spare);
        qq = reinterpret_cast<typename WK::Q *>(q32 + (warp * SM::G + g) * QCAP_T);
        cw = reinterpret_cast<typename WK::C *>(reinterpret_cast<int2 *>(q32 + NG * QCAP_T) + (warp * SM::G + g) * 25);
    }
    int total;  // candidates of the target
    // ---- the 25 stencil columns as ranges of the record arrays, with their
    // prefix.  Without PSE (which sums every candidate of the 5x5x5 cells) the
    // cells that lie wholly beyond the target's support radius are left out
    // (org.w = the margin in cells, 0 = off; org.xyz = the grid origin of this
    // step's hash): in cell units, a column's x-y box and a cell's z extent,
    // each widened by the margin, against the sphere of radius 2h around the
    // target.  Only
    // out-of-support candidates go, in the same order, so the in-support
    // queue and every sum over it are unchanged.  Cell 0 of an axis also holds
    // positions up to one cell below the origin (the hash truncates toward 0).
    constexpr bool PRUNE = COND != MFREE_COND_PSE;
    const float4 org = PRUNE ? sm.org : make_float4(0.f, 0.f, 0.f, 0.f);
    float ux = 0.f, uy = 0.f, uz = 0.f, rc2 = 0.f;
    if (PRUNE && org.w != 0.f) {
        const float ic = 1.0f / P.gdx;
        ux = (I.x - org.x) * ic;
        uy = (I.y - org.y) * ic;
        uz = (I.z - org.z) * ic;
        const float rc = 2.0f * I.h * ic;
        rc2 = rc * rc;
    }
    {
        const int klo = max(gk - 2, 0), khi = min(gk + 2, nz - 1);
        constexpr int NSET = (25 + LPP - 1) / LPP;
        int carry = 0;
#pragma unroll
        for (int k = 0; k < NSET; k++) {
            const int c = sl + k * LPP;
            int b = 0, l = 0;
            if (valid && c < 25) {
                const int cx = gi + c / 5 - 2, cy = gj + c % 5 - 2;
                if (cx >= 0 && cx < nx && cy >= 0 && cy < ny) {
                    int k0 = klo, k1 = khi;
                    if (PRUNE && org.w != 0.f) {
                        const float mg = org.w;
                        const float lox = (cx == 0 ? -1.f : float(cx)) - mg;
                        const float loy = (cy == 0 ? -1.f : float(cy)) - mg;
                        const float ex = fmaxf(0.f, fmaxf(lox - ux, ux - (float(cx + 1) + mg)));
                        const float ey = fmaxf(0.f, fmaxf(loy - uy, uy - (float(cy + 1) + mg)));
                        const float d2 = ex * ex + ey * ey;
                        if (d2 < rc2) {
                            const float zr = sqrtf(rc2 - d2) + mg;
                            int z1 = int(floorf(uz + zr));
                            if (z1 < 0 && uz + zr > -1.f) z1 = 0;
                            k0 = max(k0, int(floorf(uz - zr)));
                            k1 = min(k1, z1);
                        } else {
                            k1 = k0 - 1;
                        }
                    }
                    if (k1 >= k0) {
                        const int lc = (cx - X0 + 2) * HY + (cy - Y0 + 2);
                        const int s0 = sm.cellstart[lc][k0 - zl];
                        l = sm.cellstart[lc][k1 + 1 - zl] - s0;
                        b = STAGED ? sm.hoff[lc] + (s0 - sm.hstart[lc]) : s0;
                    }
                }
            }
            const int inc = group_scan<LPP>(l, sl);
            if (c < 25) cw[c] = WK::pack(carry + inc, b - (carry + inc - l));
            carry += __shfl_sync(0xffffffffu, inc, (g * LPP) + LPP - 1);
        }
        total = carry;
    }
    __syncwarp();
    // ---- candidates: lane sl takes candidates sl, sl + LPP, ... of the
    // flattened stencil (consecutive lanes read consecutive records); the
    // column it is in is kept in registers and reloaded only on a crossing
    int maxtotal = total;
#pragma unroll
    for (int o = 16; o >= LPP; o >>= 1) maxtotal = max(maxtotal, __shfl_xor_sync(0xffffffffu, maxtotal, o));
    auto scan = [&](auto &&fn) {
        int col = 0;
        typename WK::C w = cw[0];
        int cend = WK::end(w), base = WK::off(w);
#pragma unroll 2
        for (int k0 = 0; k0 < maxtotal; k0 += LPP) {
            const int k = k0 + sl;
            const bool act = k < total;
            if (act) {
                while (k >= cend) {  // k < total keeps col <= 24
                    col++;
                    w = cw[col];
                    cend = WK::end(w);
                    base = WK::off(w);
                }
            }
            int j = base + k;
            if (act && !bounds_ok(a.clk, j, rstride)) j = 0;
            fn(j, act);
        }
    };
    // ---- pass A: support test, PSE, queue
    const float pse_k = -1.44269504088896341f * I.h1 * I.h1;  // exp(-r^2/h^2) = 2^(pse_k r^2)
    const float four_h2 = __fmul_rn(__fmul_rn(4.0f, I.h), I.h);
    int qn = 0;  // in-support neighbours of the target (the group's ballots: the same in every lane)
    float pse = 0.f;
    {   // two candidates per lane and iteration (k and k + LPP): both column
        // walks, then both loads, then the arithmetic, so the shared-memory
        // round trips overlap; the ballots keep the flattened order
        int col = 0;
        typename WK::C w = cw[0];
        int cend = WK::end(w), base = WK::off(w);
#pragma unroll 1
        for (int k0 = 0; k0 < maxtotal; k0 += 2 * LPP) {
            const int ka = k0 + sl, kb = ka + LPP;
            const bool acta = ka < total, actb = kb < total;
            int ja = 0, jb = 0;
            if (acta) {
                while (ka >= cend) {
                    col++;
                    w = cw[col];
                    cend = WK::end(w);
                    base = WK::off(w);
                }
                ja = base + ka;
                if (!bounds_ok(a.clk, ja, rstride)) ja = 0;
            }
            if (actb) {
                while (kb >= cend) {
                    col++;
                    w = cw[col];
                    cend = WK::end(w);
                    base = WK::off(w);
                }
                jb = base + kb;
                if (!bounds_ok(a.clk, jb, rstride)) jb = 0;
            }
            float4 Pa = make_float4(0.f, 0.f, 0.f, 0.f), Pb = Pa;
            float2 ta = make_float2(0.f, 0.f), tb = ta;
            if (acta) {
                Pa = rP[ja];
                if (COND == MFREE_COND_PSE) ta = reinterpret_cast<const float2 *>(&rC[ja])[1];
            }
            if (actb) {
                Pb = rP[jb];
                if (COND == MFREE_COND_PSE) tb = reinterpret_cast<const float2 *>(&rC[jb])[1];
            }
            bool insa = false, insb = false;
            if (acta) {
                const float r2 = dist2_rn(I.x - Pa.x, I.y - Pa.y, I.z - Pa.z);
                insa = !(r2 >= four_h2) && (r2 > 9.99999994e-9f);
                if (COND == MFREE_COND_PSE) {
                    float e2;
                    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e2) : "f"(pse_k * r2));
                    pse = fmaf((ta.x - I.T) * ta.y, e2, pse);
                }
            }
            if (actb) {
                const float r2 = dist2_rn(I.x - Pb.x, I.y - Pb.y, I.z - Pb.z);
                insb = !(r2 >= four_h2) && (r2 > 9.99999994e-9f);
                if (COND == MFREE_COND_PSE) {
                    float e2;
                    asm("ex2.approx.ftz.f32 %0, %1;" : "=f"(e2) : "f"(pse_k * r2));
                    pse = fmaf((tb.x - I.T) * tb.y, e2, pse);
                }
            }
            const unsigned ma = __ballot_sync(0xffffffffu, insa) & gmask;
            const unsigned mb = __ballot_sync(0xffffffffu, insb) & gmask;
            const int qa = qn + __popc(ma & lt_mask), qb = qn + __popc(ma) + __popc(mb & lt_mask);
            if (insa && qa < QCAP_T) qq[qa] = ja;
            if (insb && qb < QCAP_T) qq[qb] = jb;
            qn += __popc(ma) + __popc(mb);
        }
    }
    if (COND == MFREE_COND_PSE) {  // the PSE sum waits in the target's result slot
#pragma unroll
        for (int o = LPP / 2; o >= 1; o >>= 1) pse += __shfl_xor_sync(0xffffffffu, pse, o);
        if (sl == 0 && valid) sm.res[tt][18] = pse;
    }
    __syncwarp();
    const int qv = min(qn, QCAP_T);
    int maxq = qv;
#pragma unroll
    for (int o = 16; o >= LPP; o >>= 1) maxq = max(maxq, __shfl_xor_sync(0xffffffffu, maxq, o));
    const bool overflow = __any_sync(0xffffffffu, qn > QCAP_T);
    // in-support neighbours beyond the queue: found again by the same scan
    auto for_overflow = [&](auto &&fn) {
        int ord = 0;
        scan([&](int j, bool act) {
            bool ins = false;
            if (act && qn > QCAP_T) {
                const float4 Pj = rP[j];
                ins = in_support(dist2_rn(I.x - Pj.x, I.y - Pj.y, I.z - Pj.z), I.h);
            }
            const unsigned m = __ballot_sync(0xffffffffu, ins) & gmask;
            const int pos = ord + __popc(m & lt_mask);
            if (ins && pos >= QCAP_T) fn(j);
            ord += __popc(m);
        });
    };
    // ---- CSPM matrix over the in-support neighbours (interactions_gpu.cu:227-295)
    float invB[6] = {1.f, 1.f, 1.f, 0.f, 0.f, 0.f};
    if (CSPM) {
        float Bm[6];  // xx, yy, zz, xy, xz, yz
#pragma unroll
        for (int k = 0; k < 6; k++) Bm[k] = 0.f;
        // one neighbour's term: B += sv d (x) d with sv = -V_j dfac
        auto bvals = [&](const float4 Pj, float vj) {
            if (I.tool == 1.f || Pj.w == 1.f) return;
            const float dx = I.x - Pj.x, dy = I.y - Pj.y, dz = I.z - Pj.z;
            float w, dfac;
            spline(dist2_rn(dx, dy, dz), I.h1, I.fac, w, dfac);
            const float sv = -vj * dfac;
            const float tx = sv * dx, ty = sv * dy, tz = sv * dz;
            Bm[0] = fmaf(tx, dx, Bm[0]);
            Bm[1] = fmaf(ty, dy, Bm[1]);
            Bm[2] = fmaf(tz, dz, Bm[2]);
            Bm[3] = fmaf(tx, dy, Bm[3]);
            Bm[4] = fmaf(tx, dz, Bm[4]);
            Bm[5] = fmaf(ty, dz, Bm[5]);
        };
        auto bterm = [&](int j) { bvals(rP[j], rC[j].w); };
        // two queue entries per lane and iteration (q and q + LPP): both loads
        // before either term, so the shared-memory round trips overlap; each
        // lane still adds its terms in queue order
#pragma unroll 1
        for (int q0 = 0; q0 < maxq; q0 += 2 * LPP) {
            const int qa = q0 + sl, qb = qa + LPP;
            const bool a = qa < qv, b = qb < qv;
            const int ja = a ? qq[qa] : 0, jb = b ? qq[qb] : 0;
            float4 Pa = make_float4(0.f, 0.f, 0.f, 0.f), Pb = Pa;
            float va = 0.f, vb = 0.f;
            if (a) { Pa = rP[ja]; va = rC[ja].w; }
            if (b) { Pb = rP[jb]; vb = rC[jb].w; }
            if (a) bvals(Pa, va);
            if (b) bvals(Pb, vb);
        }
        if (overflow) for_overflow(bterm);
#pragma unroll
        for (int o = LPP / 2; o >= 1; o >>= 1)
#pragma unroll
            for (int k = 0; k < 6; k++) Bm[k] += __shfl_xor_sync(0xffffffffu, Bm[k], o);
        const float det = det3s(Bm);
        if (det > 9.99999994e-9f) inv3s(Bm, det, invB);
    }
    // ---- pair body over the in-support neighbours
    float acc[25];
#pragma unroll
    for (int k = 0; k < 25; k++) acc[k] = 0.f;
    const PairConst PC{P.inv_wdeltap, P.av_eta * P.av_eta, P.av_alpha, P.av_beta, P.wdeltap > 0.f};
    auto pterm = [&](int j) { pair_body<CSPM, COND>(PC, I, invB, rP[j], rV[j], rA[j], rB[j], rR[j], rC[j], acc); };
    for (int q0 = 0; q0 < maxq; q0 += LPP) {
        const int q = q0 + sl;
        if (q < qv) pterm(qq[q]);
    }
    if (overflow) for_overflow(pterm);
    {   // the target's own sigma and R: sigma_i sum g + R_i sum fab g, in each lane
        const float4 Ai = rA[si], Bi = rB[si], Ri = rR[si], Ci = rC[si];
        acc[9] = fmaf(Ai.x, acc[19], fmaf(Ai.w, acc[20], fmaf(Bi.x, acc[21], acc[9])));
        acc[10] = fmaf(Ai.w, acc[19], fmaf(Ai.y, acc[20], fmaf(Bi.y, acc[21], acc[10])));
        acc[11] = fmaf(Bi.x, acc[19], fmaf(Bi.y, acc[20], fmaf(Ai.z, acc[21], acc[11])));
        acc[9] = fmaf(Ri.x, acc[22], fmaf(Ri.w, acc[23], fmaf(Ci.x, acc[24], acc[9])));
        acc[10] = fmaf(Ri.w, acc[22], fmaf(Ri.y, acc[23], fmaf(Ci.y, acc[24], acc[10])));
        acc[11] = fmaf(Ci.x, acc[22], fmaf(Ci.y, acc[23], fmaf(Ri.z, acc[24], acc[11])));
    }
    constexpr int NACC = COND == MFREE_COND_PSE ? 18 : 19;  // (slot 18 holds the PSE sum already)
#pragma unroll
    for (int o = LPP / 2; o >= 1; o >>= 1) {
#pragma unroll
        for (int k = 0; k < NACC; k++) acc[k] += __shfl_xor_sync(0xffffffffu, acc[k], o);
    }
    if (sl == 0 && valid) {
        float *rs = sm.res[tt];
#pragma unroll
        for (int k = 0; k < NACC; k++) rs[k] = acc[k];
        rs[19] = __int_as_float(qn);
    }
    __syncwarp();
}

// threads at or above PRO_FIRST never run the epilogue (TCAP <= PRO_FIRST):
// while the others finish the current tile, they prepare the next one
constexpr int PRO_FIRST = TCAP;
__device__ __forceinline__ void pro_sync(int nthreads) { asm volatile("bar.sync 1, %0;" ::"r"(nthreads) : "memory"); }

__device__ __forceinline__ void cp_async8(void *dst, const void *src) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\ncp.async.commit_group;" ::"r"(smem_u32(dst)), "l"(src)
                 : "memory");
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;" ::: "memory"); }

// Run by the prologue threads: takes the next entry of the tile list (the
// non-empty tiles of every scene), copies its scene's arguments into the
// second args buffer when the scene is not the current tile's (busy_scene),
// builds its halo cell starts, its target ranges (read from the halo table:
// the target columns are halo columns) and halo offsets, and issues its
// staging copies.  The prepared tile is left in sm.tile / sm.scene (scene < 0:
// none left).  Once its copies are issued, each call claims the list entry of
// the next call and starts fetching it into shared memory: the claim's round
// trip then overlaps the copies, and neither it nor the entry's load waits in
// the next call (a global atomic still in flight holds up the barrier that
// follows it until it is performed).  The target table and the halo table are
// built by two warps at once, the halo table with one scan (lane l owns halo
// columns 2l and 2l + 1; the staged order of the columns is free).  The caller
// guarantees that nothing reads the staged records or the tile tables any
// more.  Kept out of line: inlined into the kernel's loop it made the pair
// rounds about 7% slower (measured on the 1M-particle step).
template <int LPP, int W, int CAP>
__device__ __noinline__ void prepare_tile(const BatchTable &T, TileSmem<LPP, W> &sm, StepArgs *sa, float4 *sarr,
                                          int busy_scene) {
    constexpr int PT = W * 32 - PRO_FIRST;
    const int ptid = threadIdx.x - PRO_FIRST, pl = ptid & 31, pw = ptid >> 5;
    for (;;) {
        if (ptid == 0) {
            int2 e = make_int2(0, -1);
            if (sm.pre_ok) {
                cp_async_wait_all();
                e = sm.pre_entry;
            } else {  // the first call, or after an empty entry (none are listed; kept for safety)
                const int k = atomicAdd(T.tile_next, 1);
                if (k < sm.list_n) e = T.tile_list[k];
            }
            sm.pre_ok = 0;
            sm.ntile = e.x;
            sm.nscene = e.y;
        }
        pro_sync(PT);
        const int t = sm.ntile, s = sm.nscene;
        if (s < 0) {
            if (ptid == 0) sm.scene = -1;
            return;
        }
        // another scene's arguments go to the second buffer (the current
        // tile's, in the first, are in use); the main loop moves them over
        const int buf = s == busy_scene ? 0 : 1;
        if (buf == 1 && sm.next_args != s) {
            const StepArgs *a0 = T.args + 2 * s;
            const int4 *src = reinterpret_cast<const int4 *>(a0 + (a0->clk->parity & 1));
            int4 *d = reinterpret_cast<int4 *>(sa + 1);
            for (int k = ptid; k < int(sizeof(StepArgs) / 16); k += PT) d[k] = src[k];
            pro_sync(PT);
            if (ptid == 0) sm.next_args = s;
        }
        const StepArgs &a = sa[buf];
        const Params &P = a.p;
        const int nx = P.gnx, ny = P.gny, nz = P.gnz;
        const TileGeo G = tile_geo(P, t);
        const int *__restrict__ first = a.s.first;
        {  // halo cell starts, each thread's loads in flight together
            constexpr int NCS = (NHC * CSROW + PT - 1) / PT;
            int csv[NCS];
#pragma unroll
            for (int r = 0; r < NCS; r++) {
                const int e = ptid + r * PT;
                const int c = e / CSROW, k = e - c * CSROW;
                const int cx = G.X0 - 2 + c / HY, cy = G.Y0 - 2 + c % HY;
                csv[r] = 0;
                if (e < NHC * CSROW && k < G.nzr && cx >= 0 && cx < nx && cy >= 0 && cy < ny) {
                    const long long fi = (long long)(cx * ny + cy) * nz + G.zl + k;
                    if (bounds_ok(a.clk, fi, (long long)P.num_cell + 1)) csv[r] = first[fi];
                }
            }
#pragma unroll
            for (int r = 0; r < NCS; r++) {
                const int e = ptid + r * PT;
                if (e < NHC * CSROW) (&sm.cellstart[0][0])[e] = csv[r];
            }
        }
        pro_sync(PT);
        if (pw == 0) {
            // target column ranges (cells Z0 .. Z0 + depth - 1 of the 16
            // target columns) and their prefix
            int len = 0;
            if (pl < NTC) {
                const int cx = G.X0 + pl / TY, cy = G.Y0 + pl % TY;
                int s0 = 0;
                if (cx < nx && cy < ny && G.Z0 < nz) {
                    const int lc = (pl / TY + 2) * HY + (pl % TY + 2);
                    s0 = sm.cellstart[lc][G.Z0 - G.zl];
                    len = sm.cellstart[lc][min(G.Z0 + P.tile_z - 1, nz - 1) + 1 - G.zl] - s0;
                }
                sm.tstart[pl] = s0;
            }
            const int ti = group_scan<32>(len, pl);
            if (pl < NTC) sm.tpref[pl] = ti - len;
            if (pl == 31) sm.tpref[NTC] = ti;
        } else if (pw == 1) {
            // the 64 halo columns (lane pl: columns 2 pl and 2 pl + 1), their
            // staged offsets and the staging decision; the tile's target count
            // (the same ranges as warp 0's) decides whether copies follow
            int ntg = 0;
            if (pl < NTC) {
                const int cx = G.X0 + pl / TY, cy = G.Y0 + pl % TY;
                if (cx < nx && cy < ny && G.Z0 < nz) {
                    const int lc = (pl / TY + 2) * HY + (pl % TY + 2);
                    ntg = sm.cellstart[lc][min(G.Z0 + P.tile_z - 1, nz - 1) + 1 - G.zl] -
                          sm.cellstart[lc][G.Z0 - G.zl];
                }
            }
            ntg = __reduce_add_sync(0xffffffffu, ntg);
            int len2[2];
#pragma unroll
            for (int h = 0; h < 2; h++) {
                const int c = 2 * pl + h;
                const int cx = G.X0 - 2 + c / HY, cy = G.Y0 - 2 + c % HY;
                const bool in = cx >= 0 && cx < nx && cy >= 0 && cy < ny;
                len2[h] = in ? sm.cellstart[c][G.nzr - 1] - sm.cellstart[c][0] : 0;
                sm.hstart[c] = sm.cellstart[c][0];
                // bounds-checked build: a column whose range lies outside
                // the record arrays is counted and not staged (len 0)
                if (!range_ok(a.clk, sm.hstart[c], len2[h], P.n_init)) len2[h] = 0;
                sm.hlen[c] = len2[h];
            }
            const int v = len2[0] + len2[1];
            const int inc = group_scan<32>(v, pl);
            sm.hoff[2 * pl] = inc - v;
            sm.hoff[2 * pl + 1] = inc - v + len2[0];
            const int tot = __shfl_sync(0xffffffffu, inc, 31);
            if (pl == 0) {
                sm.total = tot;
                sm.staged = tot <= CAP ? 1 : 0;
                if (ntg > 0 && sm.staged && tot > 0)
                    mbar_expect(&sm.bar, unsigned(tot) * unsigned(REC_N * sizeof(float4)) + unsigned(P.stage_extra));
            }
        }
        pro_sync(PT);
        if (sm.tpref[NTC] == 0) continue;  // an empty tile: take the next
        if (sm.staged && sm.total > 0) {
            // two copies a column: its P records to sarr, the interleaved rest
            // to sarr + CAP (the record arrays are one allocation: P from
            // f[REC_P], the rest from f[REC_P] + n_init)
            const float4 *gbase = a.r.f[REC_P];
            for (int q = ptid; q < 2 * NHC; q += PT) {
                const int k = q / NHC, c = q - k * NHC;
                const int len = sm.hlen[c];
                const int w = k == 0 ? 1 : REC_X;
                const size_t src = (k == 0 ? 0 : size_t(P.n_init)) + size_t(sm.hstart[c]) * w;
                const int dst = (k == 0 ? 0 : CAP) + sm.hoff[c] * w;
                if (len > 0) bulk_to_smem(sarr + dst, gbase + src, unsigned(len * w) * unsigned(sizeof(float4)), &sm.bar);
            }
        }
        if (ptid == 0) {
            sm.tile = t;
            sm.scene = s;
            const int k = atomicAdd(T.tile_next, 1);  // the next call's entry
            if (k < sm.list_n) cp_async8(&sm.pre_entry, T.tile_list + k);
            else sm.pre_entry = make_int2(0, -1);
            sm.pre_ok = 1;
        }
        return;
    }
}

template <class SM> __device__ __forceinline__ void init_tile_smem(SM &sm) {
    if (threadIdx.x == 0) {
        mbar_init(&sm.bar, 1);
        sm.parity = 0;
        sm.next_args = -1;
        sm.pre_ok = 0;
    }
    fence_proxy_async();
    __syncthreads();
}

// Persistent (one block per SM) over the tiles of every scene of the table
// (one queue).  Per tile: wait for its staged halo, then the targets in passes
// of TCAP (rounds of all warps, then the epilogue by the threads below
// PRO_FIRST); during the last pass's epilogue the threads from PRO_FIRST on
// already prepare the next tile and start its staging copies.
template <int LPP, bool CSPM, int COND, bool PREC>
__global__ void __launch_bounds__(tile_threads<CSPM>(), 1) kb_interact(BatchTable T) {
    constexpr int TILE_THREADS = tile_threads<CSPM>();
    constexpr int TILE_WARPS = TILE_THREADS / 32;
    constexpr int W = TILE_WARPS;
    constexpr int CAP = rec_capacity<LPP, W>();
    constexpr int G = 32 / LPP;
    static_assert(TILE_THREADS - PRO_FIRST >= 64, "the prologue needs two warps at least");
    extern __shared__ __align__(128) unsigned char dyn[];
    TileSmem<LPP, W> &sm = *reinterpret_cast<TileSmem<LPP, W> *>(dyn);
    StepArgs *sa = reinterpret_cast<StepArgs *>(dyn + args_offset<LPP, W>());
    float4 *sarr = reinterpret_cast<float4 *>(dyn + rec_offset<LPP, W>());
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int g = lane / LPP, sl = lane - g * LPP;
    if (threadIdx.x == 0) sm.list_n = *T.tile_count;
    init_tile_smem(sm);
    int cur = -1;
    if (threadIdx.x >= PRO_FIRST) prepare_tile<LPP, W, CAP>(T, sm, sa, sarr, cur);
    const StepArgs &a = sa[0];
    for (;;) {
        __syncthreads();  // the prepared tile's descriptor and tables are visible
        const int s = sm.scene;
        if (s < 0) break;
        const int tile = sm.tile;
        if (s != cur) {  // a new scene: its arguments wait in the second buffer
            const int4 *src = reinterpret_cast<const int4 *>(sa + 1);
            int4 *d = reinterpret_cast<int4 *>(sa);
            for (int k = threadIdx.x; k < int(sizeof(StepArgs) / 16); k += blockDim.x) d[k] = src[k];
            __syncthreads();
            cur = s;
        }
        const TileGeo geo = tile_geo(a.p, tile);
        const int X0 = geo.X0, Y0 = geo.Y0, zl = geo.zl;
        const float4 *gbase = a.r.f[REC_P];  // tiles read from global memory: P, then the interleaved rest
        const int gstride = a.p.n_init;
        const int ntg = sm.tpref[NTC];
        const bool staged = sm.staged != 0;
        if (threadIdx.x == 0) {  // read by the targets after the next barrier
            float4 org = make_float4(0.f, 0.f, 0.f, 0.f);
            const float md = __uint_as_float(a.clk->max_disp);
            if (!a.p.full_stencil && md <= PRUNE_DISP_MAX) {
                const float *gm = a.p.grid_moving ? a.clk->grid_min : a.p.grid_min0;
                org = make_float4(gm[0], gm[1], gm[2], md + PRUNE_SLACK);
            }
            sm.org = org;
        }
        if (staged && sm.total > 0) {
            const unsigned par = unsigned(sm.parity);
            const long long t_wait = clock64();
            bool ok = true;
            while (!mbar_try(&sm.bar, par)) {
                if (clock64() - t_wait > WAIT_CYCLES) {
                    ok = false;
                    break;
                }
            }
            if (!__syncthreads_and(ok)) {
                // the copies did not complete in time: count it (the host
                // reports MFREE_ERR_TIMEOUT), wait once more (bounded) for the
                // copies in flight to land, and leave the kernel
                if (threadIdx.x == 0) atomicAdd(&a.clk->staging_timeouts, 1);
                const long long t2 = clock64();
                while (!mbar_try(&sm.bar, par) && clock64() - t2 <= WAIT_CYCLES) {
                }
                cp_async_wait_all();  // the prologue's fetch of the next list entry
                return;
            }
            if (threadIdx.x == 0) sm.parity ^= 1;
        }
        // PSE: every term carries T_j - T_i, so when all staged records of the
        // tile hold the same temperature (and finite positions and volumes)
        // each term is exactly +0 and so is every target's sum; such a tile runs
        // the variant without conduction terms, on the pruned stencil, with the
        // same results.  The test reads the staged halo after the wait.
        bool pse_zero = false;
        if (COND == MFREE_COND_PSE && staged && sm.total > 0 && !a.p.full_stencil) {
            const float4 *rc = sarr + CAP + (REC_C - 1), *rp = sarr;
            const float T0 = rc[0].z;
            bool u = true;
            for (int k = threadIdx.x; k < sm.total; k += TILE_THREADS) {
                const float4 c = rc[k * REC_X], p = rp[k];
                u = u && c.z == T0 && isfinite(c.w) && isfinite(p.x) && isfinite(p.y) && isfinite(p.z);
            }
            pse_zero = __syncthreads_and(u) != 0;
            if (pse_zero && threadIdx.x == 0) atomicAdd(&a.clk->pse_zero_targets, (unsigned long long)ntg);
        }
        for (int t0 = 0; t0 < ntg; t0 += TCAP) {
            const int tn = min(TCAP, ntg - t0);
            const bool last = t0 + TCAP >= ntg;
            for (int tt = threadIdx.x; tt < tn; tt += TILE_THREADS) {
                const int tg = t0 + tt;
                int c = 0;
                while (c < NTC - 1 && sm.tpref[c + 1] <= tg) c++;
                int i = sm.tstart[c] + (tg - sm.tpref[c]);
                if (!bounds_ok(a.clk, i, a.p.n_init)) i = 0;
                sm.tgt[tt] = i;
                // its cell: the z row of its column whose range holds i (the
                // rows up to the tile's last target cell are in the table)
                const int *cs = sm.cellstart[(c / TY + 2) * HY + (c % TY + 2)];
                int k = geo.Z0 - zl;
                while (cs[k + 1] <= i) k++;
                sm.tcell[tt] = (c << 16) | (zl + k);
            }
            __syncthreads();
            // rounds of TILE_WARPS * G targets; a last round with few targets
            // left uses more lanes per target so fewer warps idle at the barrier
            int done = 0;
#pragma unroll 1
            while (done < tn) {
                const int rem = tn - done;
                if (LPP < 32 && rem <= TILE_WARPS) {
                    const int tt = done + warp;
                    const bool valid = tt < tn;
                    const int i = sm.tgt[valid ? tt : 0];
                    if (staged && COND == MFREE_COND_PSE && pse_zero)
                        process_target<32, CSPM, MFREE_COND_NONE, true>(a, sm, sarr, sarr, CAP, i, valid, tt, warp, 0, lane, lane, X0,
                                                             Y0, zl);
                    else if (staged)
                        process_target<32, CSPM, COND, true>(a, sm, sarr, sarr, CAP, i, valid, tt, warp, 0, lane, lane, X0,
                                                             Y0, zl);
                    else
                        process_target<32, CSPM, COND, false>(a, sm, sarr, gbase, gstride, i, valid, tt, warp, 0, lane, lane,
                                                              X0, Y0, zl);
                    done += TILE_WARPS;
                } else if (LPP < 16 && rem <= 2 * TILE_WARPS) {
                    const int g2 = lane >> 4, sl2 = lane & 15;
                    const int tt = done + warp * 2 + g2;
                    const bool valid = tt < tn;
                    const int i = sm.tgt[valid ? tt : 0];
                    if (staged && COND == MFREE_COND_PSE && pse_zero)
                        process_target<16, CSPM, MFREE_COND_NONE, true>(a, sm, sarr, sarr, CAP, i, valid, tt, warp, g2, sl2, lane, X0,
                                                             Y0, zl);
                    else if (staged)
                        process_target<16, CSPM, COND, true>(a, sm, sarr, sarr, CAP, i, valid, tt, warp, g2, sl2, lane, X0,
                                                             Y0, zl);
                    else
                        process_target<16, CSPM, COND, false>(a, sm, sarr, gbase, gstride, i, valid, tt, warp, g2, sl2, lane,
                                                              X0, Y0, zl);
                    done += 2 * TILE_WARPS;
                } else {
                    const int tt = done + warp * G + g;
                    const bool valid = tt < tn;
                    const int i = sm.tgt[valid ? tt : 0];
                    if (staged && COND == MFREE_COND_PSE && pse_zero)
                        process_target<LPP, CSPM, MFREE_COND_NONE, true>(a, sm, sarr, sarr, CAP, i, valid, tt, warp, g, sl, lane, X0,
                                                              Y0, zl);
                    else if (staged)
                        process_target<LPP, CSPM, COND, true>(a, sm, sarr, sarr, CAP, i, valid, tt, warp, g, sl, lane, X0,
                                                              Y0, zl);
                    else
                        process_target<LPP, CSPM, COND, false>(a, sm, sarr, gbase, gstride, i, valid, tt, warp, g, sl, lane,
                                                               X0, Y0, zl);
                    done += TILE_WARPS * G;
                }
            }
            // the rounds were the last generic reads of the staged halo and the
            // tile tables: order them before the next tile's bulk writes, which
            // the prologue threads issue after this barrier
            fence_proxy_async();
            __syncthreads();
            if (threadIdx.x < PRO_FIRST) {
                if (threadIdx.x < tn) epilogue<PREC, COND>(a, sm.tgt[threadIdx.x], sm.res[threadIdx.x]);
            } else if (last) {
                prepare_tile<LPP, W, CAP>(T, sm, sa, sarr, s);
            }
            if (!last) __syncthreads();
        }
    }
}

// ------------------------------------------------------------ dispatch --
template <int LPP, bool CSPM, int COND, bool PREC> struct Variant {
    static cudaError_t batch(const BatchTable &T, int grid, cudaStream_t s) {
        auto kern = kb_interact<LPP, CSPM, COND, PREC>;
        if (grid <= 0)  // prepare only: raise the shared-memory limit (outside any graph capture)
            return cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, SMEM_LIMIT);
        kern<<<grid, tile_threads<CSPM>(), SMEM_LIMIT, s>>>(T);
        return cudaGetLastError();
    }
};

// calls fn(Variant<LPP, ...>{}) for the variant of the options
template <int LPP, class F> static cudaError_t with_variant(bool cspm, int cond, bool prec, F &&fn) {
#define MFREE_CASE(C, CO, PR) \
    if (cspm == C && cond == CO && prec == PR) return fn(Variant<LPP, C, CO, PR>{});
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

template <class F> static cudaError_t with_lpp(int lpp, bool cspm, int cond, bool prec, F &&fn) {
    switch (lpp) {
        case 8: return with_variant<8>(cspm, cond, prec, fn);
        case 16: return with_variant<16>(cspm, cond, prec, fn);
        case 32: return with_variant<32>(cspm, cond, prec, fn);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace mfree
