// elemental_kernel.cuh -- fused FP64 HDG elemental kernel for sm_100a (the kernel template and its
// launcher; elemental.cu dispatches, elemental_inst_*.cu instantiate the launchers per shape).
//
// One CTA per element (persistent grid-stride over elements), every intermediate in shared
// memory.  Replaces the reference's chunked pipeline
//   kernel/hdg_elemental.m:45-203 -> volint.m (volgeom.m) -> faceint.m (facegeom.m)
//   -> schur_primal.m:52-150 (schur_uq2; C twin kernel/schur_uq.c:42-191)
// and returns the same four arrays [AE, FE, DUDG, DUDG_DUH] in the same layouts.
//
// The algebra is the reference's, reorganised so that the two big coupling operators are
// never formed:
//   * B = dRu/dq (BD(:,:,:,ncu+1:end)) only enters through B Mi C, B Mi E and B Mi Rq.  With
//     B = sum_g sum_i shapvg(r,g,i) shapvt(g,s) wrl_i(g,a,(b,d)) (+ face terms), these become
//     sum_g sum_i shapvg(r,g,i) sum_d wrl_i(g,a,(b,d)) Z(g,.,d) where Z is Mi C / Mi E / Mi Rq
//     interpolated to the Gauss points (sum factorisation; cf. the BMiCvol/BMiCface
//     experiments at kernel/hdg_elemental.m:206-520).
//   * GK = dRh/d(u,q) is applied to DUDG and DUDG_DUH at the face Gauss points:
//     (GK X)(a,(n,j)) = sum_g shapfg(n,g) jac_g sum_c FHu(g,a,c) sum_m shapft(g,m) X(perm(m,j),c).
// H is face-block diagonal and is added directly.  Results equal the reference's up to
// floating-point summation order.
#pragma once
#include <cuda_runtime.h>
#include <atomic>
#include <type_traits>
#include <math.h>
#include "hdgx_common.cuh"
#include "tcgen05.cuh"

namespace hdgx {

struct ElemParams {
    const double *shapvt, *shapvg, *shapmv, *shapft, *shapfg, *shapmf;
    const int *perm;
    PhysConst pc;
    FbouConst fb;              // boundary-flux family and constants (fbou.m of the app's physics)
    double fc_q, fc_u;
    int tdep;                  // 1: time-dependent source s = SH_u - fc_u u (volint.m:180-221)
    int nbnd;
    int bcm[HDGX_MAX_BND];
    double bcs[HDGX_MAX_BND * 5];
    int ne;
    const double *dgnodes, *UDG, *UH, *SH;
    const int *bf;
    double *AE, *FE, *DUDG, *DUDG_DUH;
    int *status;
    double *QDG;               // non-NULL: getq mode (kernel/getq.m), the element stops after inv(M)
    int nco;                   // components stored in DUDG / DUDG_DUH: nc, or ncu when app.getdqdg = 0
    double *RU;                // non-NULL: residual mode (kernel/cuda_residual.m), Ru at q = getq(u, uh)
    double *ws;                // global workspace of plans beyond shared memory (set by the launcher)
};

// One launch over the same-shape elements of several independent element sets (e.g. of several
// serving requests): segment s is seg[s]'s arrays and physics, its elements are
// [seg_start[s], seg_start[s + 1]) of the launch; the master tables are seg[0]'s.  The table is the
// kernel's parameter (up to 32 KB of parameters on sm_70+ with CUDA 12.1+), so a launch needs no
// upload and is captured into a CUDA graph like any other.
constexpr int kMaxSeg = 24;
struct SegTable {
    ElemParams seg[kMaxSeg];
    int seg_start[kMaxSeg + 1];
    int nseg;
};
static_assert(sizeof(SegTable) < 32000, "kernel parameter limit");

// The launch's base parameters (the master tables) and its element count
__device__ __forceinline__ const ElemParams &base_params(const ElemParams &A) { return A; }
__device__ __forceinline__ const ElemParams &base_params(const SegTable &A) { return A.seg[0]; }
__device__ __forceinline__ int launch_ne(const ElemParams &A) { return A.ne; }
__device__ __forceinline__ int launch_ne(const SegTable &A) { return A.seg_start[A.nseg]; }

template <int ND_, int NPV_, int NPF_, int NGV_, int NGF_>
struct Dims {
    static constexpr int ND = ND_, NPV = NPV_, NPF = NPF_, NGV = NGV_, NGF = NGF_;
    static constexpr int NFE = ND + 1, NCU = ND + 2, NC = NCU * (ND + 1);
    static constexpr int NDF = NPF * NFE, NU = NPV * NCU, NQ = NPV * NC, NH = NCU * NDF;
    static constexpr int NGT = NGF * NFE;
};

// Shared-memory plan (in doubles).  "P" = persistent through the element, "X" = the
// assembly-phase scratch, reused by the DUDG_DUH / AE column tiles at the end.  The scratch
// is ordered so that everything the SD build does not read comes first (dead once the
// right-hand sides and Rh are built); when it is large enough SD is built on top of it
// (SD_ALIAS), and in the mixed form the FP32 inverse of SD follows it (the rest of the scratch
// is dead during the solve).  The geometry tables shapmv / shapmf are read from global
// memory (L1) instead: they are used once per element.  Less shared memory per element means
// more elements resident per SM (the kernel is latency-bound).
constexpr int al16(int x) { return (x + 15) / 16 * 16; }   // a double offset rounded up to 128 bytes

// Placement of the tensor-core operands of the mixed form in the free scratch ranges
// [x_start, inv_lo) and [inv_hi, x_end) (double offsets): A (SD^-1, adbl doubles) and a B tile of
// nbuf B tiles of nb right-hand sides each (nb a multiple of 16 dividing np).  The widest nb
// that fits is taken (every MMA round costs two CTA barriers and a proxy fence; measured on 3D
// p = 2: four rounds of 32 right-hand sides beat eight double-buffered rounds of 16), with a
// second buffer when two tiles of that width fit.  pl 0: no placement.
struct TcPlace {
    int pl, nb, nbuf, a, b;
};
constexpr TcPlace tc_place(bool mixed, int x_start, int inv_lo, int inv_hi, int x_end, int adbl, int kc, int np) {
    if (!mixed) return {0, 16, 1, 0, 0};
    for (int nb = np; nb >= 16; nb -= 16)
        for (int nbuf = 2; nbuf >= 1; nbuf--) {
            if (np % nb || nb > 256 || (nbuf == 2 && nb == np)) continue;   // two buffers need two rounds
            const int bdbl = nbuf * al16(2 * (nb / 8) * kc * 128 / 8);
            if (al16(al16(inv_hi) + adbl) + bdbl <= x_end) return {1, nb, nbuf, al16(inv_hi), al16(al16(inv_hi) + adbl)};
            if (al16(x_start) + adbl <= inv_lo && al16(inv_hi) + bdbl <= x_end)
                return {2, nb, nbuf, al16(x_start), al16(inv_hi)};
            if (al16(inv_hi) + adbl <= x_end && al16(x_start) + bdbl <= inv_lo)
                return {3, nb, nbuf, al16(inv_hi), al16(x_start)};
        }
    return {0, 16, 1, 0, 0};
}

template <class D, bool VISC, bool MIXED = false, bool TAB = true>
struct Plan {
    // master tables (loaded once per CTA; shapvt / shapvg stay in global memory when !TAB)
    static constexpr bool TABLES = TAB;
    static constexpr int t_vt = 0;
    static constexpr int t_vg = t_vt + (TAB ? D::NGV * D::NPV * (D::ND + 1) : 0);
    static constexpr int t_ft = t_vg + (TAB ? D::NPV * D::NGV * (D::ND + 1) : 0);
    static constexpr int t_fg = t_ft + D::NGF * D::NPF;
    // assembly scratch, first group: not read by the SD build
    static constexpr int x_start = t_fg + D::NPF * D::NGF;
    static constexpr int x_Xx = x_start;                          // [NGV, ND, ND]
    static constexpr int x_jac = x_Xx + D::NGV * D::ND * D::ND;
    static constexpr int x_nl = x_jac + D::NGV;                   // [NGT, ND]
    static constexpr int x_jf = x_nl + D::NGT * D::ND;
    static constexpr int x_ug = x_jf + D::NGT;                    // [NGV, NC]
    static constexpr int x_fu = x_ug + D::NGV * D::NC;            // [NGT, NC]
    static constexpr int x_fuh = x_fu + D::NGT * D::NC;           // [NGT, NCU]
    static constexpr int x_wrk = x_fuh + D::NGT * D::NCU;         // [NGV, ND, NCU]
    static constexpr int x_FH = x_wrk + D::NGV * D::ND * D::NCU;  // [NGT, NCU] jac*fhat
    static constexpr int x_BH = x_FH + D::NGT * D::NCU;           // [NGT, NCU] jac*(fbou or fhat)
    static constexpr int x_FHh = x_BH + D::NGT * D::NCU;          // [NGT, NCU, NCU] jac*dfhat/duh
    static constexpr int x_Ze = x_FHh + D::NGT * D::NCU * D::NCU; // [NGV, NDF, ND]
    static constexpr int x_Zr = x_Ze + (VISC ? D::NGV * D::NDF * D::ND : 0);   // [NGV, NCU, ND]
    static constexpr int x_ZFe = x_Zr + (VISC ? D::NGV * D::NCU * D::ND : 0);  // [NGT, NDF, ND]
    static constexpr int x_ZFr = x_ZFe + (VISC ? D::NGT * D::NDF * D::ND : 0); // [NGT, NCU, ND]
    static constexpr int p_M = x_ZFr + (VISC ? D::NGT * D::NCU * D::ND : 0);   // mass matrix (dead after inv(M))
    static constexpr int x_dead_end = p_M + D::NPV * D::NPV;
    // second group: read by the SD build
    static constexpr int x_wrl = x_dead_end;                      // [NGV, ND, NCU, NC]
    static constexpr int x_FHu = x_wrl + D::NGV * D::ND * D::NCU * D::NC;  // [NGT, NCU, NC] jac*dfhat/dudg
    static constexpr int x_Zc = x_FHu + D::NGT * D::NCU * D::NC;  // [NGV, NPV, ND]
    static constexpr int x_ZFc = x_Zc + (VISC ? D::NGV * D::NPV * D::ND : 0);  // [NGT, NPV, ND]
    static constexpr int x_end = x_ZFc + (VISC ? D::NGT * D::NPV * D::ND : 0);
    static constexpr int x_size = x_end - x_start;
    static constexpr bool SD_ALIAS = D::NU * D::NU <= x_dead_end - x_start;
    static constexpr bool INV_ALIAS = MIXED && (SD_ALIAS ? 2 : 1) * D::NU * D::NU <= x_size;
    // persistent per element
    static constexpr int p_dg = x_end;
    static constexpr int p_udg = p_dg + D::NPV * D::ND;
    static constexpr int p_uh = p_udg + D::NPV * D::NC;
    static constexpr int p_R = p_uh + D::NCU * D::NDF;            // [NU, 1+NH]
    static constexpr int p_MiC = p_R + D::NU * (1 + D::NH);       // [NPV, NPV*ND] | MiE | MiRq contiguous
    static constexpr int p_MiE = p_MiC + D::NPV * D::NPV * D::ND;
    static constexpr int p_MiRq = p_MiE + D::NPV * D::NDF * D::ND;
    static constexpr int p_Gp = p_MiRq + D::NPV * D::NCU * D::ND; // [NGT, NCU, NC] jac * dRh-flux/dudg
    static constexpr int p_Hp = p_Gp + D::NGT * D::NCU * D::NC;   // [NGT, NCU, NCU] jac * dRh-flux/duh
    static constexpr int p_Rh = p_Hp + D::NGT * D::NCU * D::NCU;
    static constexpr int p_dudg = p_Rh + D::NH;
    static constexpr int p_jv = p_dudg + D::NQ;                   // [NGV] volume jac (time-dependent mass term)
    static constexpr int p_SDsep = p_jv + D::NGV;                 // SD when it does not fit the scratch
    static constexpr int p_end = p_SDsep + (SD_ALIAS ? 0 : D::NU * D::NU);
    static constexpr int p_SD = SD_ALIAS ? x_start : p_SDsep;
    // column tiles of DUDG_DUH (reuse the scratch)
    static constexpr int NCG = VISC ? D::NC : D::NCU;
    static constexpr int per_col = D::NQ + D::NGT * NCG + D::NGT * D::NCU;
    static constexpr int TILE_RAW = x_size / per_col;
    static constexpr int TILE = TILE_RAW < 1 ? 1 : (TILE_RAW > D::NH ? D::NH : TILE_RAW);
    static constexpr int y_X = x_start;
    static constexpr int y_Xg = y_X + D::NQ * TILE;
    static constexpr int y_Y = y_Xg + D::NGT * NCG * TILE;
    static constexpr int y_end = y_Y + D::NGT * D::NCU * TILE;
    static_assert(y_end <= x_end, "the column tiles fit the scratch");
    static constexpr int d_slots = p_end;                               // 3 x u64 pivot slots
    static constexpr int d_pcol = d_slots + 4;                          // [4*NU] pivot column copies
    static constexpr int d_diag = d_pcol + 4 * D::NU;                   // [NU] pivots
    static constexpr int d_b0 = d_diag + D::NU;                         // [NU] first right-hand side
    static constexpr int d_invsep = d_b0 + D::NU;                       // [NU*NU] FP32-accurate SD^-1 (MIXED)
    static constexpr int d_mbar = d_invsep + ((MIXED && !INV_ALIAS) ? D::NU * D::NU : 0);   // tensor-core mbarrier
    static constexpr int n_doubles_core = d_mbar + (MIXED ? 4 : 0);               // two mbarriers (16-byte slot each)
    static constexpr int d_inv = INV_ALIAS ? x_start + (SD_ALIAS ? D::NU * D::NU : 0) : d_invsep;
    // Tensor-core Schur product of the mixed form, X = SD^-1 [B Mi E - F] (tcgen05, 3xTF32): the
    // operands, SD^-1 as A (M = 128 rows of which NU are real, K = NU padded to the MMA step) and
    // 16 right-hand-side columns at a time as B (N = 16), are staged in shared memory that is dead
    // once the residual column has passed its check: the assembly scratch outside SD^-1 (SD itself
    // is no longer read).  The A descriptor covers 16 row groups; the rows past NU are never
    // used, but they must lie inside the CTA's shared memory.
    static constexpr int TC_KP = (D::NU + 7) / 8 * 8;                     // K, a multiple of 8
    static constexpr int TC_KC = TC_KP / 4;                               // 16-byte K chunks per row group
    static constexpr int TC_G = (D::NU + 7) / 8;                          // row groups of A with real rows
    static constexpr int TC_NP = (D::NH + 15) / 16 * 16;                  // right-hand sides, padded
    static constexpr int TC_ADBL = 2 * TC_G * TC_KC * 128 / 8;            // A hi + lo, in doubles
    static constexpr int inv_lo = INV_ALIAS ? d_inv : x_end, inv_hi = INV_ALIAS ? d_inv + D::NU * D::NU : x_end;
    static constexpr TcPlace TCP = tc_place(MIXED, x_start, inv_lo, inv_hi, x_end, TC_ADBL, TC_KC, TC_NP);
    static constexpr int TC_PL = TCP.pl, TC_NB = TCP.nb, TC_NBUF = TCP.nbuf, tc_a = TCP.a, tc_b = TCP.b;
    static constexpr int TC_BSTRIDE = al16(2 * (TC_NB / 8) * TC_KC * 128 / 8);   // doubles between B tiles
    // integers (after the doubles in shared memory)
    static constexpr int i_perm = 0;                      // [NPF, NFE] 0-based
    static constexpr int i_invp = D::NPF * D::NFE;        // [NPV, NFE] face-local index or -1
    static constexpr int i_piv = i_invp + D::NPV * D::NFE;
    static constexpr int i_pivM = i_piv + D::NU;
    static constexpr int i_rowused = i_pivM + D::NPV;
    static constexpr int i_rowvar = i_rowused + D::NU;
    static constexpr int i_gslot = i_rowvar + D::NU;
    static constexpr int i_bf = i_gslot + 2;
    static constexpr int i_bad = i_bf + D::NFE;
    static constexpr int i_tmem = i_bad + 1;              // TMEM address of the tensor-core accumulator
    static constexpr int n_ints = i_tmem + 1;
    // Plans beyond a CTA's shared memory (3D p = 3: 520 KB for 100 unknowns and 201 right-hand
    // sides) keep every double array in a per-CTA slice of a global workspace, read and written
    // through L1 and L2 (one CTA per SM), with the integers in shared memory; the local system is
    // then LU-factored and solved in shared memory (below).
    static constexpr bool WS = sizeof(double) * n_doubles_core + sizeof(int) * n_ints > 227 * 1024;
    static constexpr int n_doubles = n_doubles_core;
    static constexpr int ws_stride = al16(n_doubles);                       // doubles per CTA slice
    static constexpr bool TC = !WS && TC_PL != 0 && tc_a * 8 + 16 * TC_KC * 128 <= (int)(sizeof(double) * n_doubles) &&
                               TC_NP <= 256 && D::NU <= 64;
    static constexpr size_t bytes = sizeof(double) * n_doubles + sizeof(int) * n_ints;   // the whole plan
    // WS shared memory, in doubles after the integers: the face tables t_ft / t_fg (ws_tabs), SD
    // (built there and LU-factored in place, at lu_off) followed by the right-hand sides solved in
    // LU_NCH chunks of LU_CH columns (leading dimension NU + 1 against bank conflicts); before the
    // SD build the same space holds the first scratch group [x_start, x_dead_end) (ws_dead: on
    // top of SD when SD is built over that group, else after it)
    static constexpr int ws_tabs = al16((n_ints * (int)sizeof(int) + 7) / 8);
    static constexpr int lu_off = al16(ws_tabs + 2 * D::NGF * D::NPF);
    static constexpr int ws_dead = SD_ALIAS ? lu_off : lu_off + D::NU * D::NU;
    static constexpr int LU_CHMAX = (227 * 1024 / 8 - lu_off - D::NU * D::NU) / (D::NU + 1);
    static constexpr int LU_NCH = (1 + D::NH + LU_CHMAX - 1) / (LU_CHMAX > 0 ? LU_CHMAX : 1);
    static constexpr int LU_CH = (1 + D::NH + LU_NCH - 1) / LU_NCH;
    static constexpr int ws_smem_doubles = (lu_off + D::NU * D::NU + (D::NU + 1) * LU_CH) >
                                                   (ws_dead + x_dead_end - x_start)
                                               ? lu_off + D::NU * D::NU + (D::NU + 1) * LU_CH
                                               : ws_dead + x_dead_end - x_start;
    static constexpr size_t smem_bytes = WS ? sizeof(double) * ws_smem_doubles : bytes;   // of it in shared memory
    static_assert(!WS || LU_CHMAX >= 1, "the LU factors and one column fit shared memory");
    static_assert(!WS || smem_bytes <= 227 * 1024, "the shared-memory part of the plan fits");
};

// Resident elements per SM: the kernel is latency-bound (barrier-separated phases, a 40-step
// elimination), so more elements in flight per SM beat more threads per element.  A plan that
// fits four CTAs per SM runs four of 128 threads, one that fits three runs three of 192 (up to
// 112 registers each); the larger plans run two or one of 256.  (C2, 2D NS p = 3: 6.84 ms
// with two CTAs of 256, 6.21 ms with three of 192; 2D p = 2: 3.01 -> 1.80 ms with four of 128.)
// The volume tables shapvt / shapvg move from shared to global memory (read through L1) only
// when that raises the number of resident CTAs (2D p = 4: 119 -> 108 KB, one -> two per SM).
constexpr int blocks_for(size_t bytes) {
    return bytes <= 45 * 1024 ? 4 : (bytes <= 74 * 1024 ? 3 : (bytes <= 110 * 1024 ? 2 : 1));
}
template <class D, bool VISC, bool MIXED>
using PlanSel = Plan<D, VISC, MIXED,
                     (!Plan<D, VISC, MIXED, false>::WS &&
                      blocks_for(Plan<D, VISC, MIXED, false>::bytes) <= blocks_for(Plan<D, VISC, MIXED, true>::bytes))>;
template <class D, bool VISC, bool MIXED>
constexpr int min_blocks() { return blocks_for(PlanSel<D, VISC, MIXED>::bytes); }
template <class D, bool VISC, bool MIXED>
constexpr int cta_threads() {
    return PlanSel<D, VISC, MIXED>::WS ? 512
                                       : (min_blocks<D, VISC, MIXED>() == 4 ? 128
                                                                            : (min_blocks<D, VISC, MIXED>() == 3 ? 192 : 256));
}

// MIXED: the local elimination of the Jacobian columns runs in FP32 (with the identity
// appended so that the FP32 inverse of SD comes out too); the local residual solve (DUDG)
// is then refined against the FP64 SD to FP64 accuracy, and every residual (Ru, Rq, Rh, FE)
// is FP64.  AE and DUDG_DUH therefore carry FP32-level errors (a Jacobian error, which
// changes the Newton convergence rate, not the converged solution).
// Tensor-core Schur product also in plans that run several CTAs per SM (see USE_TC below).
constexpr bool kTcMultiCta = false;

template <class D, bool VISC, bool MIXED, int NT, class Arg = ElemParams>
__global__ void __launch_bounds__(NT, (min_blocks<D, VISC, MIXED>())) elemental_kernel(const __grid_constant__ Arg A) {
    constexpr bool SEG = !std::is_same<Arg, ElemParams>::value;
    const ElemParams &P = base_params(A);
    using L = PlanSel<D, VISC, MIXED>;
    constexpr int ND = D::ND, NPV = D::NPV, NPF = D::NPF, NGV = D::NGV, NGF = D::NGF;
    constexpr int NFE = D::NFE, NCU = D::NCU, NC = D::NC, NDF = D::NDF, NU = D::NU;
    constexpr int NQ = D::NQ, NH = D::NH, NGT = D::NGT;
    constexpr int NSEED = VISC ? NC : NCU;   // inviscid flux does not depend on q
    constexpr int NCG = VISC ? NC : NCU;     // components dRh/dudg couples (q-part is 0 for Euler)
    extern __shared__ __align__(16) double sm[];
    // the doubles of the plan: shared memory, or this CTA's slice of the global workspace
    double *wk = L::WS ? P.ws + (size_t)blockIdx.x * L::ws_stride : sm;
    int *si = L::WS ? reinterpret_cast<int *>(sm) : reinterpret_cast<int *>(sm + L::n_doubles);
    const int tid = threadIdx.x;

    const double *t_vt = L::TABLES ? wk + L::t_vt : P.shapvt, *t_vg = L::TABLES ? wk + L::t_vg : P.shapvg;
    // WS: the face tables, SD and the first scratch group in shared memory (see Plan)
    double *smd = reinterpret_cast<double *>(sm);
    double *t_ft = L::WS ? smd + L::ws_tabs : wk + L::t_ft, *t_fg = L::WS ? t_ft + NGF * NPF : wk + L::t_fg;
    double *xd = L::WS ? smd + L::ws_dead - L::x_start : wk;     // base of the first scratch group
    const double *__restrict__ t_mv = P.shapmv;   // geometry tables: read once per element from L1
    const double *__restrict__ t_mf = P.shapmf;
    int *perm = si + L::i_perm, *invp = si + L::i_invp;

    // ---- master tables, once per CTA
    if constexpr (L::TABLES) {
        for (int i = tid; i < NGV * NPV * (ND + 1); i += NT) {
            wk[L::t_vt + i] = P.shapvt[i];
            wk[L::t_vg + i] = P.shapvg[i];
        }
    }
    for (int i = tid; i < NGF * NPF; i += NT) {
        t_ft[i] = P.shapft[i];   // value slice of shapft[ngf,npf,nd]
        t_fg[i] = P.shapfg[i];   // value slice of shapfg[npf,ngf,nd]
    }
    for (int i = tid; i < NPF * NFE; i += NT) perm[i] = P.perm[i] - 1;
    for (int i = tid; i < NPV * NFE; i += NT) invp[i] = -1;
    __syncthreads();
    for (int i = tid; i < NPF * NFE; i += NT) invp[perm[i] + NPV * (i / NPF)] = i % NPF;
    // mixed form: the tensor-memory accumulator of the Schur product and its mbarrier, once per CTA
    constexpr uint32_t TC_COLS = L::TC_NP <= 32 ? 32 : (L::TC_NP <= 64 ? 64 : (L::TC_NP <= 128 ? 128 : 256));
    // Kernels that hold tensor memory run one CTA per SM (the runtime limits a TMEM-allocating
    // kernel's occupancy to 1), while the smaller plans run three or four elements per SM and
    // are bound by the latency of their elimination chain: the tensor-core Schur product is used
    // where the plan runs one CTA per SM anyway (3D p = 2).
    constexpr bool USE_TC = L::TC && (min_blocks<D, VISC, MIXED>() == 1 || kTcMultiCta);
    uint64_t *s_mbar = reinterpret_cast<uint64_t *>(wk + L::d_mbar);
    uint32_t tmem = 0, tc_phases = 0;          // bit b: the phase parity mbarrier b waits for next
    if constexpr (USE_TC) {
        if (tid < 32) tc::tmem_alloc<TC_COLS>(reinterpret_cast<uint32_t *>(si + L::i_tmem));
        if (tid == 0) {
            tc::mbar_init(s_mbar, 1);
            tc::mbar_init(s_mbar + 2, 1);
            asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
        }
        tc::fence_before_sync();
    }
    __syncthreads();
    if constexpr (USE_TC) {
        tc::fence_after_sync();
        tmem = *reinterpret_cast<const uint32_t *>(si + L::i_tmem);
    }

    double *s_dg = wk + L::p_dg, *s_udg = wk + L::p_udg, *s_uh = wk + L::p_uh;
    double *s_SD = L::WS ? smd + L::lu_off : wk + L::p_SD, *s_R = wk + L::p_R;
    double *s_MiC = wk + L::p_MiC, *s_MiE = wk + L::p_MiE, *s_MiRq = wk + L::p_MiRq;
    double *s_Gp = wk + L::p_Gp, *s_Hp = wk + L::p_Hp, *s_Rh = wk + L::p_Rh, *s_M = xd + L::p_M;
    double *s_dudg = wk + L::p_dudg, *s_jv = wk + L::p_jv;
    double *x_Xx = xd + L::x_Xx, *x_jac = xd + L::x_jac, *x_nl = xd + L::x_nl, *x_jf = xd + L::x_jf;
    double *x_ug = xd + L::x_ug, *x_fu = xd + L::x_fu, *x_fuh = xd + L::x_fuh;
    double *x_wrk = xd + L::x_wrk, *x_wrl = wk + L::x_wrl, *x_FH = xd + L::x_FH, *x_BH = xd + L::x_BH;
    double *x_FHu = wk + L::x_FHu, *x_FHh = xd + L::x_FHh;
    double *x_Zc = wk + L::x_Zc, *x_Ze = xd + L::x_Ze, *x_Zr = xd + L::x_Zr;
    double *x_ZFc = wk + L::x_ZFc, *x_ZFe = xd + L::x_ZFe, *x_ZFr = xd + L::x_ZFr;
    int *s_piv = si + L::i_piv, *s_pivM = si + L::i_pivM, *s_bf = si + L::i_bf, *s_bad = si + L::i_bad;
    int *s_rowused = si + L::i_rowused, *s_rowvar = si + L::i_rowvar, *s_gslot = si + L::i_gslot;
    unsigned long long *s_slot = reinterpret_cast<unsigned long long *>(wk + L::d_slots);
    double *s_pcol = wk + L::d_pcol, *s_diag = wk + L::d_diag;

    int seg = 0;                                 // segmented launches: the segment of element eg
    const int ne_launch = launch_ne(A);
    for (int eg = blockIdx.x; eg < ne_launch; eg += gridDim.x) {
        const ElemParams *Qp = &P;
        int e = eg;
        if constexpr (SEG) {
            while (eg >= A.seg_start[seg + 1]) seg++;
            Qp = &A.seg[seg];
            e = eg - A.seg_start[seg];
        }
        const ElemParams &Q = *Qp;   // this element's arrays and physics
        bool force_piv = false;      // set when the unpivoted solve failed its check and SD sits on
                                     // the scratch: the element is then evaluated again, pivoted
    elem_start:
        // ================================================================ load
        {
            const double *g_dg = Q.dgnodes + (size_t)e * NPV * ND;
            const double *g_udg = Q.UDG + (size_t)e * NPV * NC;
            const double *g_uh = Q.UH + (size_t)e * NCU * NDF;
            for (int i = tid; i < NPV * ND; i += NT) s_dg[i] = g_dg[i];
            for (int i = tid; i < NPV * NC; i += NT) s_udg[i] = g_udg[i];
            for (int i = tid; i < NCU * NDF; i += NT) s_uh[i] = g_uh[i];
            if (tid < NFE) s_bf[tid] = Q.bf[(size_t)e * NFE + tid];
            if (tid == 0) *s_bad = 0;
        }
        __syncthreads();

        // ====================================================== geometry, traces
        // volgeom.m:18-61 (Jg(k,m) = dx_m/dxi_k; Xx = adj(Jg)); facegeom.m:20-52.
        for (int g = tid; g < NGV; g += NT) {
            double J[ND][ND];
#pragma unroll
            for (int k = 0; k < ND; k++)
#pragma unroll
                for (int m = 0; m < ND; m++) {
                    double t = 0.0;
#pragma unroll
                    for (int n = 0; n < NPV; n++) t += t_mv[g + NGV * (n + NPV * (k + 1))] * s_dg[n + NPV * m];
                    J[k][m] = t;
                }
            double *X = x_Xx + g;   // X(i,j) at X[NGV*(i + ND*j)]
            if constexpr (ND == 2) {
                x_jac[g] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
                X[NGV * (0 + 2 * 0)] = J[1][1];
                X[NGV * (1 + 2 * 0)] = -J[1][0];
                X[NGV * (0 + 2 * 1)] = -J[0][1];
                X[NGV * (1 + 2 * 1)] = J[0][0];
            } else {
                x_jac[g] = J[0][0] * J[1][1] * J[2][2] - J[0][0] * J[2][1] * J[1][2] + J[1][0] * J[2][1] * J[0][2]
                         - J[1][0] * J[0][1] * J[2][2] + J[2][0] * J[0][1] * J[1][2] - J[2][0] * J[1][1] * J[0][2];
                X[NGV * (0 + 3 * 0)] = J[1][1] * J[2][2] - J[1][2] * J[2][1];
                X[NGV * (1 + 3 * 0)] = J[1][2] * J[2][0] - J[1][0] * J[2][2];
                X[NGV * (2 + 3 * 0)] = J[1][0] * J[2][1] - J[1][1] * J[2][0];
                X[NGV * (0 + 3 * 1)] = J[0][2] * J[2][1] - J[0][1] * J[2][2];
                X[NGV * (1 + 3 * 1)] = J[0][0] * J[2][2] - J[0][2] * J[2][0];
                X[NGV * (2 + 3 * 1)] = J[0][1] * J[2][0] - J[0][0] * J[2][1];
                X[NGV * (0 + 3 * 2)] = J[0][1] * J[1][2] - J[0][2] * J[1][1];
                X[NGV * (1 + 3 * 2)] = J[0][2] * J[1][0] - J[0][0] * J[1][2];
                X[NGV * (2 + 3 * 2)] = J[0][0] * J[1][1] - J[0][1] * J[1][0];
            }
        }
        for (int gg = tid; gg < NGT; gg += NT) {
            const int g = gg % NGF, j = gg / NGF;
            double dp[ND][ND > 1 ? ND - 1 : 1];
#pragma unroll
            for (int m = 0; m < ND; m++)
#pragma unroll
                for (int k = 0; k < ND - 1; k++) {
                    double t = 0.0;
#pragma unroll
                    for (int n = 0; n < NPF; n++)
                        t += t_mf[g + NGF * (n + NPF * (k + 1))] * s_dg[perm[n + NPF * j] + NPV * m];
                    dp[m][k] = t;
                }
            if constexpr (ND == 2) {
                const double jc = sqrt(dp[0][0] * dp[0][0] + dp[1][0] * dp[1][0]);
                x_jf[gg] = jc;
                x_nl[gg + NGT * 0] = dp[1][0] / jc;
                x_nl[gg + NGT * 1] = -dp[0][0] / jc;
            } else {
                const double n0 = dp[1][0] * dp[2][1] - dp[2][0] * dp[1][1];
                const double n1 = dp[2][0] * dp[0][1] - dp[0][0] * dp[2][1];
                const double n2 = dp[0][0] * dp[1][1] - dp[1][0] * dp[0][1];
                const double jc = sqrt(n0 * n0 + n1 * n1 + n2 * n2);
                x_jf[gg] = jc;
                x_nl[gg + NGT * 0] = n0 / jc;
                x_nl[gg + NGT * 1] = n1 / jc;
                x_nl[gg + NGT * 2] = n2 / jc;
            }
        }
        // volint.m:31-33 / faceint.m:55-61: solution and trace at the Gauss points
        for (int i = tid; i < NGV * NC; i += NT) {
            const int g = i % NGV, c = i / NGV;
            double t = 0.0;
#pragma unroll
            for (int n = 0; n < NPV; n++) t += t_vt[g + NGV * n] * s_udg[n + NPV * c];
            x_ug[i] = t;
        }
        for (int i = tid; i < NGT * NC; i += NT) {
            const int gg = i % NGT, c = i / NGT, g = gg % NGF, j = gg / NGF;
            double t = 0.0;
#pragma unroll
            for (int n = 0; n < NPF; n++) t += t_ft[g + NGF * n] * s_udg[perm[n + NPF * j] + NPV * c];
            x_fu[i] = t;
        }
        for (int i = tid; i < NGT * NCU; i += NT) {
            const int gg = i % NGT, a = i / NGT, g = gg % NGF, j = gg / NGF;
            double t = 0.0;
#pragma unroll
            for (int n = 0; n < NPF; n++) t += t_ft[g + NGF * n] * s_uh[a + NCU * (n + NPF * j)];
            x_fuh[i] = t;
        }
        __syncthreads();

        // ============================================= M, C, E (volint.m:43-55, faceint.m:37-48)
        for (int i = tid; i < NPV * NPV; i += NT) {
            const int r = i % NPV, s = i / NPV;
            double t = 0.0;
#pragma unroll
            for (int g = 0; g < NGV; g++) t += t_vg[r + NPV * g] * t_vt[g + NGV * s] * x_jac[g];
            s_M[i] = Q.fc_q * t;
        }
        if (tid < NGV) s_jv[tid] = x_jac[tid];
        for (int i = tid; i < NPV * NPV * ND; i += NT) {
            const int r = i % NPV, s = (i / NPV) % NPV, d = i / (NPV * NPV);
            double t = 0.0;
#pragma unroll
            for (int g = 0; g < NGV; g++) {
                double w = 0.0;
#pragma unroll
                for (int jd = 0; jd < ND; jd++) w += t_vg[r + NPV * (g + NGV * (jd + 1))] * x_Xx[g + NGV * (d + ND * jd)];
                t += w * t_vt[g + NGV * s];
            }
            s_MiC[i] = t;                          // C(r,s,d), solved in place below
        }
        for (int i = tid; i < NPV * NDF * ND; i += NT) {
            const int r = i % NPV, f = (i / NPV) % NDF, d = i / (NPV * NDF);
            const int n = f % NPF, j = f / NPF, m = invp[r + NPV * j];
            double t = 0.0;
            if (m >= 0) {
#pragma unroll
                for (int g = 0; g < NGF; g++) {
                    const int gg = g + NGF * j;
                    t += t_fg[m + NPF * g] * t_ft[g + NGF * n] * x_nl[gg + NGT * d] * x_jf[gg];
                }
            }
            s_MiE[i] = t;                          // E(r,(n,j),d)
        }
        __syncthreads();
        // Rq = M (SH/fc_q - q) + C u - E uh   (volint.m:57-60, faceint.m:49-51)
        const double *__restrict__ g_shq = Q.SH + (size_t)e * NPV * NC + NPV * NCU;   // q part of SH
        for (int i = tid; i < NPV * NCU * ND; i += NT) {
            const int r = i % NPV, a = (i / NPV) % NCU, d = i / (NPV * NCU);
            const int cq = NCU + a + NCU * d;
            double t = 0.0;
#pragma unroll
            for (int s = 0; s < NPV; s++)
                t += s_M[r + NPV * s] * ((Q.SH ? g_shq[s + NPV * (a + NCU * d)] / Q.fc_q : 0.0) -
                                         ((Q.QDG || Q.RU) ? 0.0 : s_udg[s + NPV * cq]));   // getq: q does not enter
#pragma unroll
            for (int s = 0; s < NPV; s++) t += s_MiC[r + NPV * (s + NPV * d)] * s_udg[s + NPV * a];
            for (int f = 0; f < NDF; f++) t -= s_MiE[r + NPV * (f + NDF * d)] * s_uh[a + NCU * f];
            s_MiRq[i] = t;
        }
        __syncthreads();

        // ============================ Mi = inv(M): MiC, MiE, MiRq (schur_primal.m:86-91)
        // M is SPD (exact quadrature of phi phi jac): eliminate without pivoting
        gj_regs_nopiv<NPV, NPV * ND + NDF * ND + NCU * ND, NT, 8>(s_M, s_MiC, s_pcol, s_bad);
        if (tid == 0 && *s_bad) *s_bad = 1;
        __syncthreads();
        if (Q.QDG) {
            // getq.m:37-104: the q that zeroes Rq for this u and uh; with q left out of Rq above,
            // Mi Rq = inv(fc_q Mu) (fc_q Mu SH_q / fc_q + C u - E uh)
            double *g_q = Q.QDG + (size_t)e * NPV * NCU * ND;
            for (int i = tid; i < NPV * NCU * ND; i += NT) g_q[i] = s_MiRq[i];
            if (tid == 0 && Q.status) Q.status[e] = *s_bad;
            __syncthreads();
            continue;
        }
        if (Q.RU) {
            // cuda_residual.m:3-4: q from getq, then the u residual is evaluated at that q; Rq is
            // zero at that q, so Mi Rq (and its Gauss-point values below) are set to exact zeros
            for (int i = tid; i < NPV * NCU * ND; i += NT) {
                s_udg[NPV * NCU + i] = s_MiRq[i];
                s_MiRq[i] = 0.0;
            }
            __syncthreads();
            for (int i = tid; i < NGV * NCU * ND; i += NT) {
                const int g = i % NGV, c = NCU + i / NGV;
                double t = 0.0;
#pragma unroll
                for (int n = 0; n < NPV; n++) t += t_vt[g + NGV * n] * s_udg[n + NPV * c];
                x_ug[g + NGV * c] = t;
            }
            for (int i = tid; i < NGT * NCU * ND; i += NT) {
                const int gg = i % NGT, c = NCU + i / NGT, g = gg % NGF, j = gg / NGF;
                double t = 0.0;
#pragma unroll
                for (int n = 0; n < NPF; n++) t += t_ft[g + NGF * n] * s_udg[perm[n + NPF * j] + NPV * c];
                x_fu[gg + NGT * c] = t;
            }
            __syncthreads();
        }

        // ================================ flux / fhat / fbou at the Gauss points
        // volume: thread (g, seed); volint.m:81, 241-254
        for (int i = tid; i < NGV * NSEED; i += NT) {
            const int g = i % NGV, sd = i / NGV;
            D1 u[NCU], q[NCU * ND], f[NCU * ND];
#pragma unroll
            for (int c = 0; c < NCU; c++) u[c] = {x_ug[g + NGV * c], c == sd ? 1.0 : 0.0};
#pragma unroll
            for (int c = 0; c < NCU * ND; c++) q[c] = {x_ug[g + NGV * (NCU + c)], (NCU + c) == sd ? 1.0 : 0.0};
            ns_flux<ND>(Q.pc, u, q, f);
#pragma unroll
            for (int id = 0; id < ND; id++)
#pragma unroll
                for (int a = 0; a < NCU; a++) {
                    double w = 0.0, dw = 0.0;
#pragma unroll
                    for (int jd = 0; jd < ND; jd++) {
                        const double xx = x_Xx[g + NGV * (jd + ND * id)];
                        w += f[a + NCU * jd].v * xx;
                        dw += f[a + NCU * jd].d * xx;
                    }
                    if (sd == 0) x_wrk[g + NGV * (id + ND * a)] = w;
                    x_wrl[g + NGV * (id + ND * (a + NCU * sd))] = -dw;
                }
        }
        if constexpr (!VISC) {
            for (int i = tid; i < NGV * ND * NCU * (NC - NCU); i += NT) x_wrl[NGV * ND * NCU * NCU + i] = 0.0;
        }
        // faces: thread (gg, seed); fhat.m:49-67 = f(uh,q).n + tau (u - uh)
        for (int i = tid; i < NGT * NSEED; i += NT) {
            const int gg = i % NGT, sd = i / NGT;
            D1 u[NCU], q[NCU * ND], f[NCU * ND];
#pragma unroll
            for (int c = 0; c < NCU; c++) u[c] = {x_fuh[gg + NGT * c], c == sd ? 1.0 : 0.0};
#pragma unroll
            for (int c = 0; c < NCU * ND; c++) q[c] = {x_fu[gg + NGT * (NCU + c)], (NCU + c) == sd ? 1.0 : 0.0};
            ns_flux<ND>(Q.pc, u, q, f);
            const double jc = x_jf[gg];
            const int j = gg / NGF;
            const int bnd = s_bf[j] < 0;
            const int ib = bnd ? -s_bf[j] - 1 : 0;
            const int btype = bnd ? ((ib < Q.nbnd) ? Q.bcm[ib] : -1) : 0;
            const bool dir = bnd && btype == 6;                        // ns/fbou.m:111-114, both families
            const bool per = bnd && btype == 5 && Q.fb.fam == 0;       // ns/fbou.m:109-110: fhat
            const bool gen = bnd && !dir && !per;                      // the other fbou.m types
#pragma unroll
            for (int a = 0; a < NCU; a++) {
                double fn = 0.0, dfn = 0.0;
#pragma unroll
                for (int jd = 0; jd < ND; jd++) {
                    const double nl = x_nl[gg + NGT * jd];
                    fn += f[a + NCU * jd].v * nl;
                    dfn += f[a + NCU * jd].d * nl;
                }
                if (sd == 0) {
                    const double fh = fn + Q.pc.tau * (x_fu[gg + NGT * a] - x_fuh[gg + NGT * a]);
                    x_FH[gg + NGT * a] = jc * fh;
                    const double bh = dir ? (x_fuh[gg + NGT * a] - Q.bcs[ib * 5 + a]) : fh;
                    if (!gen) x_BH[gg + NGT * a] = jc * bh;
                }
                if (sd < NCU) {
                    // dfhat/duh (seed on uh) and dfhat/du = tau I
                    const double fhh = dfn - (a == sd ? Q.pc.tau : 0.0);
                    const double fhu = (a == sd ? Q.pc.tau : 0.0);
                    x_FHh[gg + NGT * (a + NCU * sd)] = jc * fhh;
                    x_FHu[gg + NGT * (a + NCU * sd)] = jc * fhu;
                    if (!gen) {
                        s_Hp[gg + NGT * (a + NCU * sd)] = jc * (dir ? (a == sd ? 1.0 : 0.0) : fhh);
                        s_Gp[gg + NGT * (a + NCU * sd)] = jc * (dir ? 0.0 : fhu);
                    }
                } else {
                    x_FHu[gg + NGT * (a + NCU * sd)] = jc * dfn;
                    if (!gen) s_Gp[gg + NGT * (a + NCU * sd)] = jc * (dir ? 0.0 : dfn);
                }
            }
            if (gen) {
                // faceint.m:171-268: Rh, H and GK rows of this boundary face from fbou.m.  One pass
                // seeded like the fhat above (uh for sd < NCU, q otherwise) and, for sd < NCU, one
                // seeded on the interior u.
                double nlp[ND];
#pragma unroll
                for (int d = 0; d < ND; d++) nlp[d] = x_nl[gg + NGT * d];
                D1 uu[NCU], qq[NCU * ND], hh[NCU], fb[NCU];
#pragma unroll
                for (int c = 0; c < NCU; c++) {
                    uu[c] = {x_fu[gg + NGT * c], 0.0};
                    hh[c] = {x_fuh[gg + NGT * c], c == sd ? 1.0 : 0.0};
                }
#pragma unroll
                for (int c = 0; c < NCU * ND; c++) qq[c] = {x_fu[gg + NGT * (NCU + c)], (NCU + c) == sd ? 1.0 : 0.0};
                const double *ub = Q.bcs + (ib < Q.nbnd ? ib : 0) * 5;
                if (!fbou_point<ND>(Q.fb, Q.pc, btype, ub, nlp, uu, qq, hh, fb)) *s_bad = 3;
#pragma unroll
                for (int a = 0; a < NCU; a++) {
                    if (sd == 0) x_BH[gg + NGT * a] = jc * fb[a].v;
                    if (sd < NCU) s_Hp[gg + NGT * (a + NCU * sd)] = jc * fb[a].d;
                    else s_Gp[gg + NGT * (a + NCU * sd)] = jc * fb[a].d;
                }
                if (sd < NCU) {
#pragma unroll
                    for (int c = 0; c < NCU; c++) {
                        uu[c].d = c == sd ? 1.0 : 0.0;
                        hh[c].d = 0.0;
                    }
                    fbou_point<ND>(Q.fb, Q.pc, btype, ub, nlp, uu, qq, hh, fb);
#pragma unroll
                    for (int a = 0; a < NCU; a++) s_Gp[gg + NGT * (a + NCU * sd)] = jc * fb[a].d;
                }
            }
        }
        if constexpr (!VISC) {
            for (int i = tid; i < NGT * NCU * (NC - NCU); i += NT) {
                x_FHu[NGT * NCU * NCU + i] = 0.0;
                s_Gp[NGT * NCU * NCU + i] = 0.0;
            }
        }
        // Mi C, Mi E, Mi Rq at the volume and face Gauss points (only B couples through them)
        if constexpr (VISC) {
            for (int i = tid; i < NGV * NPV * ND; i += NT) {
                const int g = i % NGV, kd = i / NGV;
                double t = 0.0;
#pragma unroll
                for (int s = 0; s < NPV; s++) t += t_vt[g + NGV * s] * s_MiC[s + NPV * kd];
                x_Zc[i] = t;
            }
            for (int i = tid; i < NGV * NDF * ND; i += NT) {
                const int g = i % NGV, fd = i / NGV;
                double t = 0.0;
#pragma unroll
                for (int s = 0; s < NPV; s++) t += t_vt[g + NGV * s] * s_MiE[s + NPV * fd];
                x_Ze[i] = t;
            }
            for (int i = tid; i < NGV * NCU * ND; i += NT) {
                const int g = i % NGV, bd = i / NGV;
                double t = 0.0;
#pragma unroll
                for (int s = 0; s < NPV; s++) t += t_vt[g + NGV * s] * s_MiRq[s + NPV * bd];
                x_Zr[i] = t;
            }
            for (int i = tid; i < NGT * NPV * ND; i += NT) {
                const int gg = i % NGT, kd = i / NGT, g = gg % NGF, j = gg / NGF;
                double t = 0.0;
#pragma unroll
                for (int n = 0; n < NPF; n++) t += t_ft[g + NGF * n] * s_MiC[perm[n + NPF * j] + NPV * kd];
                x_ZFc[i] = t;
            }
            for (int i = tid; i < NGT * NDF * ND; i += NT) {
                const int gg = i % NGT, fd = i / NGT, g = gg % NGF, j = gg / NGF;
                double t = 0.0;
#pragma unroll
                for (int n = 0; n < NPF; n++) t += t_ft[g + NGF * n] * s_MiE[perm[n + NPF * j] + NPV * fd];
                x_ZFe[i] = t;
            }
            for (int i = tid; i < NGT * NCU * ND; i += NT) {
                const int gg = i % NGT, bd = i / NGT, g = gg % NGF, j = gg / NGF;
                double t = 0.0;
#pragma unroll
                for (int n = 0; n < NPF; n++) t += t_ft[g + NGF * n] * s_MiRq[perm[n + NPF * j] + NPV * bd];
                x_ZFr[i] = t;
            }
        }
        __syncthreads();

        // ========================= SD = D + B Mi C (schur_primal.m:93-110 with volint/faceint)
        // One batched GEMM per (a, b) component pair over the volume (g, id) and face (j, g)
        // quadrature points kk:  SD((r,a),(k,b)) = sum_kk Phi(r, kk) W_ab(kk, k), with
        //   Phi = shapvg(r, g, id) (volume) / shapfg(m(r, j), g) (face; 0 off the face) and
        //   W_ab = wrl(g,id,a,b) shapvt(g,k) + sum_d wrl(g,id,a,(b,d)) Zc(g,k,d)           (volume)
        //        = shapft(g,n(k,j)) FHu(gg,a,b) + sum_d FHu(gg,a,(b,d)) ZFc(gg,k,d)        (face)
        // W is formed on the fly, once per register tile.
        constexpr int KV = NGV * ND, KK = KV + NFE * NGF;
        constexpr int TMS = NPV <= 6 ? NPV : (NPV + 1) / 2;
        auto phi = [&](int, int r, int kk) -> double {
            if (kk < KV) return t_vg[r + NPV * (kk + NGV)];      // shapvg(r, g, id + 1), kk = g + NGV id
            const int kf = kk - KV, j = kf / NGF, g = kf % NGF, m = invp[r + NPV * j];
            return m >= 0 ? t_fg[m + NPF * g] : 0.0;
        };
        auto build_sd = [&]() {
        tile_gemm<NCU * NCU, NPV, NPV, KK, TMS, 2, NT, 2>(
            phi,
            [&](int ab, int kk, int k) -> double {
                const int a = ab % NCU, b = ab / NCU;
                if (kk < KV) {
                    const int g = kk % NGV, id = kk / NGV;
                    double w = x_wrl[g + NGV * (id + ND * (a + NCU * b))] * t_vt[g + NGV * k];
                    if constexpr (VISC) {
#pragma unroll
                        for (int d = 0; d < ND; d++)
                            w += x_wrl[g + NGV * (id + ND * (a + NCU * (NCU + b + NCU * d)))] * x_Zc[g + NGV * (k + NPV * d)];
                    }
                    return w;
                }
                const int kf = kk - KV, j = kf / NGF, g = kf % NGF, gg = g + NGF * j, nk = invp[k + NPV * j];
                double w = nk >= 0 ? t_ft[g + NGF * nk] * x_FHu[gg + NGT * (a + NCU * b)] : 0.0;
                if constexpr (VISC) {
#pragma unroll
                    for (int d = 0; d < ND; d++)
                        w += x_FHu[gg + NGT * (a + NCU * (NCU + b + NCU * d))] * x_ZFc[gg + NGT * (k + NPV * d)];
                }
                return w;
            },
            [&](int ab, int r, int k, double v) {
                const int a = ab % NCU, b = ab / NCU;
                if (Q.tdep && a == b) {
                    // time-dependent problems: the source Jacobian -fc_u on the u components
                    // (volint.m:215-216) enters BD, hence D, as fc_u * sum_g phi_r phi_k w_g jac_g
                    double mu = 0.0;
#pragma unroll
                    for (int g = 0; g < NGV; g++) mu += t_vg[r + NPV * g] * t_vt[g + NGV * k] * s_jv[g];
                    v += Q.fc_u * mu;
                }
                s_SD[(r + NPV * a) + NU * (k + NPV * b)] = v;
            });
        };
        auto build_rhs = [&]() {
        // rhs0 = Ru - B Mi Rq (volint.m:258, faceint.m:306-331; schur_primal.m:95,111)
        for (int i = tid; i < NU; i += NT) {
            const int r = i % NPV, a = i / NPV;
            double v = 0.0;
            for (int g = 0; g < NGV; g++)
#pragma unroll
                for (int id = 0; id < ND; id++) {
                    double w = x_wrk[g + NGV * (id + ND * a)];
                    if constexpr (VISC) {
                        for (int bd = 0; bd < NCU * ND; bd++)
                            w -= x_wrl[g + NGV * (id + ND * (a + NCU * (NCU + bd)))] * x_Zr[g + NGV * bd];
                    }
                    v += t_vg[r + NPV * (g + NGV * (id + 1))] * w;
                }
#pragma unroll
            for (int j = 0; j < NFE; j++) {
                const int m = invp[r + NPV * j];
                if (m < 0) continue;
                for (int g = 0; g < NGF; g++) {
                    const int gg = g + NGF * j;
                    double w = -x_FH[gg + NGT * a];
                    if constexpr (VISC) {
                        for (int bd = 0; bd < NCU * ND; bd++)
                            w -= x_FHu[gg + NGT * (a + NCU * (NCU + bd))] * x_ZFr[gg + NGT * bd];
                    }
                    v += t_fg[m + NPF * g] * w;
                }
            }
            if (Q.tdep) {
                // s = SH_u - fc_u u at the volume Gauss points, Ru += shapvg(:,:,1) (s jac)
                // (volint.m:180-221 with dtcoef = 1 and no axisymmetry; volint.m:241,258)
                const double *__restrict__ g_sh = Q.SH ? Q.SH + (size_t)e * NPV * NC + NPV * a : nullptr;
                for (int g = 0; g < NGV; g++) {
                    double st = 0.0;
#pragma unroll
                    for (int s = 0; s < NPV; s++) st += t_vt[g + NGV * s] * (g_sh ? g_sh[s] : 0.0);
                    v += t_vg[r + NPV * g] * ((st - x_ug[g + NGV * a] * Q.fc_u) * s_jv[g]);
                }
            }
            s_R[i] = v;
        }
        // RHS((r,a), (b,f)) = B Mi E - F   (schur_primal.m:98,118; faceint.m:319-333): the same
        // batched GEMM with W_ab(kk, f) = sum_d wrl(g,id,a,(b,d)) Ze(g,f,d) (volume) and
        // sum_d FHu(gg,a,(b,d)) ZFe(gg,f,d) (face), minus the face-block F term
        tile_gemm<NCU * NCU, NPV, NDF, (VISC ? KK : 0), TMS, 2, NT, 2>(
            phi,
            [&](int ab, int kk, int f) -> double {
                const int a = ab % NCU, b = ab / NCU;
                double w = 0.0;
                if (kk < KV) {
                    const int g = kk % NGV, id = kk / NGV;
#pragma unroll
                    for (int d = 0; d < ND; d++)
                        w += x_wrl[g + NGV * (id + ND * (a + NCU * (NCU + b + NCU * d)))] * x_Ze[g + NGV * (f + NDF * d)];
                } else {
                    const int kf = kk - KV, j = kf / NGF, g = kf % NGF, gg = g + NGF * j;
#pragma unroll
                    for (int d = 0; d < ND; d++)
                        w += x_FHu[gg + NGT * (a + NCU * (NCU + b + NCU * d))] * x_ZFe[gg + NGT * (f + NDF * d)];
                }
                return w;
            },
            [&](int ab, int r, int f, double v) {
                const int a = ab % NCU, b = ab / NCU, nf = f % NPF, jf = f / NPF;
                const int mf = invp[r + NPV * jf];
                if (mf >= 0) {
                    double t = 0.0;
#pragma unroll
                    for (int g = 0; g < NGF; g++)
                        t += t_fg[mf + NPF * g] * t_ft[g + NGF * nf] * x_FHh[(g + NGF * jf) + NGT * (a + NCU * b)];
                    v -= t;
                }
                s_R[NU + (r + NPV * a) + NU * (b + NCU * f)] = v;
            });
        };
        build_rhs();
        if (Q.RU) {
            // cuda_residual.m: the element u residual Ru (volume and face terms, time source)
            __syncthreads();
            for (int i = tid; i < NU; i += NT) Q.RU[(size_t)e * NU + i] = s_R[i];
            if (tid == 0 && Q.status) Q.status[e] = *s_bad;
            __syncthreads();
            continue;
        }
        // Rh = -(fbou or fhat) integrated on each face (faceint.m:335-339)
        for (int i = tid; i < NH; i += NT) {
            const int a = i % NCU, mf = i / NCU, m = mf % NPF, j = mf / NPF;
            double t = 0.0;
            for (int g = 0; g < NGF; g++) t += t_fg[m + NPF * g] * x_BH[(g + NGF * j) + NGT * a];
            s_Rh[i] = -t;
        }
        if constexpr (L::SD_ALIAS) __syncthreads();     // SD overwrites what the RHS and Rh read
        build_sd();
        __syncthreads();

        // ================================ LU of SD and the 1 + NH solves (schur_primal.m:111,118)
        {
            int bad_before = *s_bad;
            bool tc_go = false;          // the unpivoted mixed solve passed its check: Schur product next
            __syncthreads();
            if constexpr (L::WS) {
                // LU with partial pivoting of SD in shared memory (dgesv's factorisation), then the
                // 1 + NH right-hand sides in chunks: gathered in the pivot order, forward and back
                // substitution in shared memory, the solution written straight to s_R
                constexpr int NU1 = NU + 1, CH = L::LU_CH;
                double *l_LU = s_SD, *l_B = l_LU + NU * NU;   // SD is built in shared memory: factored in place
                int *ip = s_rowvar;                      // row of SD that ends up at position i
                block_lu<NT>(l_LU, NU, NU, s_piv, s_bad);
                if (tid == 0) {
                    for (int i = 0; i < NU; i++) ip[i] = i;
                    for (int k = 0; k < NU; k++) {
                        const int q = s_piv[k], t = ip[k];
                        ip[k] = ip[q];
                        ip[q] = t;
                    }
                }
                __syncthreads();
                for (int c0 = 0; c0 < 1 + NH; c0 += CH) {
                    const int nc = (1 + NH - c0) < CH ? (1 + NH - c0) : CH;
                    for (int t = tid; t < NU * nc; t += NT) {
                        const int i = t % NU, j = t / NU;
                        l_B[i + NU1 * j] = s_R[ip[i] + NU * (c0 + j)];
                    }
                    __syncthreads();
                    for (int k = 0; k < NU - 1; k++) {       // L y = P b (unit lower triangle)
                        const int m = NU - k - 1;
                        for (int t = tid; t < m * nc; t += NT) {
                            const int i = k + 1 + t % m, j = t / m;
                            l_B[i + NU1 * j] -= l_LU[i + NU * k] * l_B[k + NU1 * j];
                        }
                        __syncthreads();
                    }
                    for (int k = NU - 1; k >= 0; k--) {      // U x = y: row k is final at step k
                        const double ukk = l_LU[k + NU * k];
                        for (int t = tid; t < (k + 1) * nc; t += NT) {
                            const int i = t % (k + 1), j = t / (k + 1);
                            const double xk = l_B[k + NU1 * j] / ukk;
                            if (i == k) s_R[k + NU * (c0 + j)] = xk;
                            else l_B[i + NU1 * j] -= l_LU[i + NU * k] * xk;
                        }
                        __syncthreads();
                    }
                }
            } else if (force_piv) {
                gj_regs<NU, 1 + NH, NT, 8, true>(s_SD, s_R, s_pcol, s_diag, s_rowvar, s_gslot, s_bad);
            } else {
            // Unpivoted elimination with the density unknowns last (in natural order interior
            // nodes have structurally zero density pivots: the continuity flux does not depend on
            // the density), accepted when the backward error of the first column,
            // |b0 - SD x0| / (|SD| |x0| + |b0|) (infinity norms), is below 1e-13; otherwise the
            // element is redone with partial pivoting in FP64.
            double *s_b0 = wk + L::d_b0;
            for (int i = tid; i < NU; i += NT) s_b0[i] = s_R[i];
            __syncthreads();
            if constexpr (MIXED) {
                // FP32 elimination of [SD | R | I] (with the tensor-core Schur product: of
                // [SD | r0 | I] only, the other right-hand sides are multiplied by SD^-1 below),
                // then the residual column refined in FP64 against the FP64 SD with the FP32 inverse
                double *s_inv = wk + L::d_inv;
                gj_regs_nopiv_t<float, NU, USE_TC ? 1 : 1 + NH, NU, true, NT, 8, NPV>(
                    s_SD, s_R, s_inv, reinterpret_cast<float *>(s_pcol), s_bad);
                double *s_res = s_pcol;                    // free after the elimination
                for (int it = 0; it < 3; it++) {
                    for (int r = tid; r < NU; r += NT) {
                        double res = s_b0[r];
#pragma unroll 8
                        for (int c = 0; c < NU; c++) res -= s_SD[r + NU * c] * s_R[c];
                        s_res[r] = res;
                    }
                    __syncthreads();
                    for (int r = tid; r < NU; r += NT) {
                        double dx = 0.0;
#pragma unroll 8
                        for (int c = 0; c < NU; c++) dx += s_inv[r + NU * c] * s_res[c];
                        s_R[r] += dx;
                    }
                    __syncthreads();
                }
            } else {
                gj_regs_nopiv<NU, 1 + NH, NT, 8, NPV>(s_SD, s_R, s_pcol, s_bad);
            }
            {
                double rmax = 0.0, amax = 0.0, xmax = 0.0, bmax = 0.0;
                for (int r = tid; r < NU; r += NT) {
                    double res = s_b0[r], as = 0.0;
                    for (int c = 0; c < NU; c++) {
                        const double sd = s_SD[r + NU * c];
                        res -= sd * s_R[c];
                        as += fabs(sd);
                    }
                    rmax = fmax(rmax, fabs(res));
                    amax = fmax(amax, as);
                    xmax = fmax(xmax, fabs(s_R[r]));
                    bmax = fmax(bmax, fabs(s_b0[r]));
                }
                if (!(rmax == rmax)) rmax = INFINITY;
                for (int o = 16; o > 0; o >>= 1) {
                    rmax = fmax(rmax, __shfl_xor_sync(0xffffffffu, rmax, o));
                    amax = fmax(amax, __shfl_xor_sync(0xffffffffu, amax, o));
                    xmax = fmax(xmax, __shfl_xor_sync(0xffffffffu, xmax, o));
                    bmax = fmax(bmax, __shfl_xor_sync(0xffffffffu, bmax, o));
                }
                double *red = s_pcol;   // free after the elimination
                if ((tid & 31) == 0) {
                    red[4 * (tid >> 5) + 0] = rmax; red[4 * (tid >> 5) + 1] = amax;
                    red[4 * (tid >> 5) + 2] = xmax; red[4 * (tid >> 5) + 3] = bmax;
                }
                __syncthreads();
                if (tid == 0) {
                    double R = 0.0, A = 0.0, X = 0.0, B = 0.0;
                    for (int w = 0; w < NT / 32; w++) {
                        R = fmax(R, red[4 * w]); A = fmax(A, red[4 * w + 1]);
                        X = fmax(X, red[4 * w + 2]); B = fmax(B, red[4 * w + 3]);
                    }
                    const double den = A * X + B;
                    const bool ok = (*s_bad == bad_before) && (R <= 1e-13 * den) && isfinite(R);
                    s_gslot[0] = ok ? 0 : 1;
                    if (!ok) *s_bad = bad_before;
                }
                __syncthreads();
            }
            tc_go = s_gslot[0] == 0;
            if (s_gslot[0]) {
                // fall back to partial pivoting on the original system
                if (L::SD_ALIAS || L::INV_ALIAS) {
                    force_piv = true;            // the right-hand sides' inputs are overwritten (by SD,
                    __syncthreads();             // or by the FP32 inverse): evaluate the element again
                    goto elem_start;
                } else {
                    build_rhs();
                    __syncthreads();
                    gj_regs<NU, 1 + NH, NT, 8, true>(s_SD, s_R, s_pcol, s_diag, s_rowvar, s_gslot, s_bad);
                }
            }
            }
            if (tid == 0 && *s_bad && !bad_before) *s_bad = 2;
            __syncthreads();
            if constexpr (USE_TC) {
                // Schur product on the tensor cores (tcgen05 kind::tf32, 3xTF32 with FP32
                // accumulation): R(:, 1:) = SD^-1 R(:, 1:) (schur_primal.m:118, dlu = SD \ (BMiE - F)),
                // once the residual column has passed its check (a pivoted redo solves R in FP64).
                // A = SD^-1 (K-major: row r, column k), B = 16 right-hand sides per MMA round (row n
                // = right-hand side, K-major), D = A B^T in TMEM columns n0 .. n0 + 15.
                if (tc_go) {
                    constexpr int KP = L::TC_KP, KC = L::TC_KC, GR = 8 * L::TC_G, NP = L::TC_NP, NB = L::TC_NB;
                    constexpr int AH = L::TC_G * KC * 128, BH = (NB / 8) * KC * 128;   // bytes of one hi / lo half
                    const double *s_inv = wk + L::d_inv;
                    unsigned char *tA = reinterpret_cast<unsigned char *>(wk + L::tc_a);
                    unsigned char *tB = reinterpret_cast<unsigned char *>(wk + L::tc_b);
                    for (int i = tid; i < GR * KP; i += NT) {
                        const int r = i % GR, k = i / GR;
                        float h = 0.f, l = 0.f;
                        if (r < NU && k < NU) tc::split_tf32(s_inv[r + NU * k], h, l);
                        const int off = tc::kmajor_offset(r, k, KC);
                        *reinterpret_cast<float *>(tA + off) = h;
                        *reinterpret_cast<float *>(tA + AH + off) = l;
                    }
                    constexpr uint32_t idesc = tc::idesc_tf32(128, NB);
                    constexpr int NBUF = L::TC_NBUF, NROUND = NP / NB;
                    const uint32_t aaddr = tc::smem_u32(tA);
                    // round r stages its B tile in buffer r % NBUF and multiplies it into TMEM columns
                    // r NB ..; buffer b's mbarrier completes once that buffer's MMAs are done, and a
                    // buffer is rewritten only after its previous round's MMAs have completed, so
                    // staging round r + 1 overlaps the tensor core's work on round r
                    for (int r = 0; r < NROUND; r++) {
                        const int b = r % NBUF, n0 = r * NB;
                        unsigned char *tb = tB + (size_t)8 * L::TC_BSTRIDE * b;
                        if (r >= NBUF) {
                            if (!tc::mbar_wait(s_mbar + 2 * b, (tc_phases >> b) & 1u, 1 << 22)) *s_bad = 4;
                            tc_phases ^= 1u << b;
                            tc::fence_after_sync();
                        }
                        for (int i = tid; i < NB * KP; i += NT) {
                            const int n = i % NB, k = i / NB;
                            float h = 0.f, l = 0.f;
                            if (n0 + n < NH && k < NU) tc::split_tf32(s_R[k + NU * (1 + n0 + n)], h, l);
                            const int off = tc::kmajor_offset(n, k, KC);
                            *reinterpret_cast<float *>(tb + off) = h;
                            *reinterpret_cast<float *>(tb + BH + off) = l;
                        }
                        tc::fence_proxy_async();
                        __syncthreads();
                        if (tid == 0) {
                            tc::fence_after_sync();
                            const uint32_t baddr = tc::smem_u32(tb);
#pragma unroll
                            for (int s = 0; s < KP / 8; s++) {
                                const uint64_t ah = tc::smem_desc(aaddr + 256 * s, 128, KC * 128);
                                const uint64_t al = tc::smem_desc(aaddr + AH + 256 * s, 128, KC * 128);
                                const uint64_t bh = tc::smem_desc(baddr + 256 * s, 128, KC * 128);
                                const uint64_t bl = tc::smem_desc(baddr + BH + 256 * s, 128, KC * 128);
                                tc::mma_tf32(tmem + n0, al, bh, idesc, s > 0);
                                tc::mma_tf32(tmem + n0, ah, bl, idesc, true);
                                tc::mma_tf32(tmem + n0, ah, bh, idesc, true);
                            }
                            tc::commit(s_mbar + 2 * b);
                        }
                    }
                    // the last round of every buffer
                    for (int b = 0; b < NBUF && b < NROUND; b++) {
                        if (!tc::mbar_wait(s_mbar + 2 * b, (tc_phases >> b) & 1u, 1 << 22)) *s_bad = 4;
                        tc_phases ^= 1u << b;
                    }
                    tc::fence_after_sync();
                    // rows r < NU are TMEM lanes 0..NU-1: warp w reads lanes 32 w .. 32 w + 31
                    if (tid < 32 * ((NU + 31) / 32)) {
                        const int w = tid >> 5;
#pragma unroll 1
                        for (int c = 0; c < NP; c += 16) {
                            float v[16];
                            tc::tmem_ld16(tmem + ((uint32_t)(32 * w) << 16) + (uint32_t)c, v);
#pragma unroll
                            for (int i = 0; i < 16; i++)
                                if (tid < NU && c + i < NH) s_R[tid + NU * (1 + c + i)] = (double)v[i];
                        }
                    }
                    tc::fence_before_sync();
                    __syncthreads();
                }
            }
        }

        // ================================ DUDG = [du, MiRq + MiC du] (schur_primal.m:112-116)
        {
            double *g_dudg = Q.DUDG + (size_t)e * NPV * Q.nco;
            for (int i = tid; i < NQ; i += NT) {
                const int r = i % NPV, c = i / NPV;
                double v;
                if (c < NCU) {
                    v = s_R[r + NPV * c];
                } else {
                    const int a = (c - NCU) % NCU, d = (c - NCU) / NCU;
                    v = s_MiRq[r + NPV * (a + NCU * d)];
#pragma unroll
                    for (int s = 0; s < NPV; s++) v += s_MiC[r + NPV * (s + NPV * d)] * s_R[s + NPV * a];
                }
                s_dudg[i] = v;
                if (c < Q.nco) g_dudg[i] = v;       // getdqdg = 0: the u rows only
            }
        }
        __syncthreads();
        // FE = Rh - GK DUDG (schur_primal.m:143-144), GK applied at the face Gauss points
        {
            double *Xg = wk + L::y_Xg;
            for (int i = tid; i < NGT * NCG; i += NT) {
                const int gg = i % NGT, c = i / NGT, g = gg % NGF, j = gg / NGF;
                double t = 0.0;
#pragma unroll
                for (int m = 0; m < NPF; m++) t += t_ft[g + NGF * m] * s_dudg[perm[m + NPF * j] + NPV * c];
                Xg[i] = t;
            }
            __syncthreads();
            double *g_fe = Q.FE + (size_t)e * NH;
            for (int i = tid; i < NH; i += NT) {
                const int a = i % NCU, nf = i / NCU, n = nf % NPF, j = nf / NPF;
                double t = 0.0;
                for (int g = 0; g < NGF; g++) {
                    const int gg = g + NGF * j;
                    double y = 0.0;
                    for (int c = 0; c < NCG; c++) y += s_Gp[gg + NGT * (a + NCU * c)] * Xg[gg + NGT * c];
                    t += t_fg[n + NPF * g] * y;
                }
                g_fe[i] = s_Rh[i] - t;
            }
            __syncthreads();
        }

        // ============ DUDG_DUH and AE = H + GK DUDG_DUH in column tiles (schur_primal.m:136-147)
        // Each column tile runs four batched small GEMMs with register tiles:
        //   X   = DUDG_DUH columns: u rows copied from the solve, q rows = MiC dlu - MiE
        //   Xg  = X at the face Gauss points (shapft through perm), per face
        //   Y   = Gp Xg, per face Gauss point (GK applied without forming it)
        //   AE  = shapfg Y (+ the face-block-diagonal H), per face
        // nco (components stored per row block) is a compile-time constant inside the tiles
        auto tiles = [&](auto nco_c) {
            constexpr int NCO = decltype(nco_c)::value;
            constexpr int T = L::TILE;
            constexpr int TMQ = NPV <= 6 ? NPV : (NPV + 1) / 2;
            double *yX = wk + L::y_X, *yXg = wk + L::y_Xg, *yY = wk + L::y_Y;
            double *g_dd = Q.DUDG_DUH + (size_t)e * NPV * NCO * NH;     // [npv, nco, ncu, ndf]
            double *g_ae = Q.AE + (size_t)e * NH * NH;
            for (int k0 = 0; k0 < NH; k0 += T) {
                const int nt = (NH - k0) < T ? (NH - k0) : T;
                for (int i = tid; i < NU * nt; i += NT) {
                    const int ru = i % NU, t = i / NU;
                    const double v = s_R[NU * (1 + k0 + t) + ru];
                    yX[ru + NQ * t] = v;
                    g_dd[(size_t)NPV * NCO * (k0 + t) + ru] = v;
                }
                // q rows r + NPV (NCU + a + NCU d) of column k = k0 + t, batch d, n = (a, t)
                tile_gemm<ND, NPV, NCU * T, NPV, TMQ, 2, NT>(
                    [&](int d, int r, int sx) { return s_MiC[r + NPV * (sx + NPV * d)]; },
                    [&](int, int sx, int n) {
                        const int t = n / NCU;
                        return t < nt ? s_R[NU * (1 + k0) + sx + NPV * n] : 0.0;
                    },
                    [&](int d, int r, int n, double v) {
                        const int a = n % NCU, t = n / NCU;
                        if (t >= nt) return;
                        const int k = k0 + t;
                        if (a == k % NCU) v -= s_MiE[r + NPV * (k / NCU + NDF * d)];
                        const int row = r + NPV * (NCU + a + NCU * d);
                        yX[row + NQ * t] = v;
                        if constexpr (NCO == NC) g_dd[(size_t)NQ * k + row] = v;
                    });
                __syncthreads();
                // Xg(gg, c, t) = sum_m shapft(g, m) X(perm(m, j), c, t), batch j, n = (c, t)
                tile_gemm<NFE, NGF, NCG * T, NPF, NGF, 2, NT>(
                    [&](int, int g, int m) { return t_ft[g + NGF * m]; },
                    [&](int j, int m, int n) {
                        const int c = n % NCG, t = n / NCG;
                        return yX[perm[m + NPF * j] + NPV * c + NQ * t];
                    },
                    [&](int j, int g, int n, double v) { yXg[g + NGF * j + NGT * n] = v; });
                __syncthreads();
                // Y(gg, a, t) = sum_c Gp(gg, a, c) Xg(gg, c, t), batch gg
                tile_gemm<NGT, NCU, T, NCG, 2, 2, NT>(
                    [&](int gg, int a, int c) { return s_Gp[gg + NGT * (a + NCU * c)]; },
                    [&](int gg, int c, int t) { return yXg[gg + NGT * (c + NCG * t)]; },
                    [&](int gg, int a, int t, double v) { yY[gg + NGT * (a + NCU * t)] = v; });
                __syncthreads();
                // AE((a, n, j), k) = sum_g shapfg(n, g) (Y(gg, a, t) + [face of k == j] shapft(g, nk) Hp(gg, a, b)),
                // batch j, rows n, columns (a, t)
                tile_gemm<NFE, NPF, NCU * T, NGF, 2, 2, NT>(
                    [&](int, int n, int g) { return t_fg[n + NPF * g]; },
                    [&](int j, int g, int nn) {
                        const int a = nn % NCU, t = nn / NCU, gg = g + NGF * j;
                        double y = yY[gg + NGT * nn];
                        const int k = k0 + t, b = k % NCU, fk = k / NCU, nk = fk % NPF, jk = fk / NPF;
                        if (t < nt && jk == j) y += t_ft[g + NGF * nk] * s_Hp[gg + NGT * (a + NCU * b)];
                        return y;
                    },
                    [&](int j, int n, int nn, double v) {
                        const int a = nn % NCU, t = nn / NCU;
                        if (t < nt) g_ae[(size_t)NH * (k0 + t) + a + NCU * (n + NPF * j)] = v;
                    });
                __syncthreads();
            }
        };
        if (Q.nco == NC) tiles(std::integral_constant<int, NC>{});
        else tiles(std::integral_constant<int, NCU>{});
        if (tid == 0 && Q.status) Q.status[e] = *s_bad;
        __syncthreads();
    }
    if constexpr (USE_TC) {
        tc::fence_before_sync();
        __syncthreads();
        if (tid < 32) tc::tmem_dealloc(tmem, TC_COLS);
    }
}

// ------------------------------------------------------------------ dispatch
inline ElemParams &base_of(ElemParams &a) { return a; }
inline ElemParams &base_of(SegTable &a) { return a.seg[0]; }

template <class D, bool VISC, bool MIXED, class Arg>
int launch_t(const Arg &p, int ne, cudaStream_t st, int grid_req) {
    constexpr int NT = cta_threads<D, VISC, MIXED>();
    using L = PlanSel<D, VISC, MIXED>;
    static_assert(L::TILE >= 1, "tile");
    const size_t smem = L::smem_bytes;
    if (smem > 227 * 1024) return -3;
    auto kern = elemental_kernel<D, VISC, MIXED, NT, Arg>;
    cudaError_t err = allow_dynamic_smem((const void *)kern, smem);
    if (err != cudaSuccess) return -10;
    // resident CTAs per SM of this instantiation, once per device
    static std::atomic<int> per_sm_cache[kMaxDevices];
    const int dev = current_device(), nsm = sm_count_of(dev);
    int per_sm = per_sm_cache[dev < kMaxDevices ? dev : 0].load(std::memory_order_relaxed);
    if (per_sm < 1) {
        // a plan in the global workspace wants the largest L1 next to its shared memory
        if (L::WS && cudaFuncSetAttribute((const void *)kern, cudaFuncAttributePreferredSharedMemoryCarveout, 0) !=
                         cudaSuccess)
            return -10;
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, NT, smem) != cudaSuccess) per_sm = 0;
        if (per_sm < 1) return -11;
        if (L::WS) per_sm = 1;                   // one CTA per SM: its slice stays in L1 / L2
        per_sm_cache[dev < kMaxDevices ? dev : 0].store(per_sm, std::memory_order_relaxed);
    }
    int grid = grid_req > 0 ? grid_req : nsm * per_sm;     // default: one wave of resident CTAs
    if (grid > ne) grid = ne;
    if (grid < 1) return 0;
    if constexpr (L::WS) {
        // the CTAs' workspace slices, from the stream-ordered allocator (freed behind the launch)
        Arg q = p;
        double *ws = nullptr;
        if (cudaMallocAsync((void **)&ws, sizeof(double) * L::ws_stride * (size_t)grid, st) != cudaSuccess)
            return -13;
        base_of(q).ws = ws;
        kern<<<grid, NT, smem, st>>>(q);
        err = cudaGetLastError();
        if (cudaFreeAsync(ws, st) != cudaSuccess && err == cudaSuccess) return -12;
    } else {
        kern<<<grid, NT, smem, st>>>(p);
        err = cudaGetLastError();
    }
    return err == cudaSuccess ? 0 : -12;
}

// The compiled element shapes: (nd, npv, npf, ngv, ngf) of 2D p = 1..4 and 3D p = 1..3 at the
// drivers' quadrature order pgauss = 2 porder.
using Tri1 = Dims<2, 3, 2, 3, 2>;
using Tri2 = Dims<2, 6, 3, 6, 3>;
using Tri3 = Dims<2, 10, 4, 12, 4>;
using Tri4 = Dims<2, 15, 5, 16, 5>;
using Tet1 = Dims<3, 4, 3, 4, 3>;
using Tet2 = Dims<3, 10, 6, 11, 6>;
using Tet3 = Dims<3, 20, 10, 24, 12>;

}  // namespace hdgx

// The launchers of one shape: FP64 and mixed, inviscid and viscous, plain and segmented (the mixed
// form of a workspace plan is not built: it runs the FP64 kernel).  EXT is `extern` for a
// declaration (elemental.cu) and empty for the definition (elemental_inst_*.cu).
#define HDGX_ELEM_LAUNCHERS_FP64(EXT, D)                                                              \
    EXT template int hdgx::launch_t<D, false, false, hdgx::ElemParams>(const hdgx::ElemParams &, int, \
                                                                       cudaStream_t, int);            \
    EXT template int hdgx::launch_t<D, true, false, hdgx::ElemParams>(const hdgx::ElemParams &, int,  \
                                                                      cudaStream_t, int);             \
    EXT template int hdgx::launch_t<D, false, false, hdgx::SegTable>(const hdgx::SegTable &, int,     \
                                                                     cudaStream_t, int);              \
    EXT template int hdgx::launch_t<D, true, false, hdgx::SegTable>(const hdgx::SegTable &, int,      \
                                                                    cudaStream_t, int);
#define HDGX_ELEM_LAUNCHERS_MIXED(EXT, D)                                                            \
    EXT template int hdgx::launch_t<D, false, true, hdgx::ElemParams>(const hdgx::ElemParams &, int, \
                                                                      cudaStream_t, int);            \
    EXT template int hdgx::launch_t<D, true, true, hdgx::ElemParams>(const hdgx::ElemParams &, int,  \
                                                                     cudaStream_t, int);
#define HDGX_ELEM_LAUNCHERS(EXT, D) HDGX_ELEM_LAUNCHERS_FP64(EXT, D) HDGX_ELEM_LAUNCHERS_MIXED(EXT, D)

