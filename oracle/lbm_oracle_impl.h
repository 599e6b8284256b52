/*
 * Oracle (test infrastructure only): CPU restatement of the reference's D3Q19
 * lattice-Boltzmann step functions.  Included twice by lbm_oracle.c, once with
 * REAL=double (the FP64 oracle) and once with REAL=float (an FP32 twin used to
 * estimate single-precision drift on the CPU).  Nothing in the product calls
 * this code; the CUDA library is checked against it.
 *
 * Reference functions restated here (paths inside yagise/MyFluidSimulation):
 *   D3Q19 tables / feq            src/lbm/lbm3d_legacy.cu:16-35,54-58
 *   equilibrium reinit            src/lbm/lbm_reinit.cu:20-50
 *   Legacy BGK collide+push       src/lbm/lbm3d_legacy.cu:59-114
 *   Hybrid(B0) collide+push       src/lbm/lbm3d_hybrid.cu:89-175
 *   HOME regularised rebuild      src/lbm/lbm3d_home.cu:37-81
 *   HOME moment-only gather step  src/lbm/lbm3d_home.cu:142-286
 *
 * Extensions with no reference counterpart (defined identically in the CUDA
 * kernels): the duct boundary (bc==1) and the momentum-exchange drag.
 *   - x is non-periodic; the link of a fluid cell that leaves through x<0 is an
 *     inlet link: the population that comes back along it is the equilibrium
 *     at (rho of the cell at this step, u=(u_in,0,0)).
 *   - a link that leaves through x>=Nx is an outlet link: the population that
 *     comes back along it equals the cell's own post-collision population in
 *     that incoming direction (zero-gradient extrapolation).
 *   - y and z stay periodic; duct walls are mask cells (value with bit 3 set,
 *     i.e. 8|1, which marks them solid but not part of the obstacle).
 *   - drag = momentum handed to obstacle cells (solid, bit 3 clear) by the
 *     populations reflected at them: (c_in - c_out) f for every reflected
 *     population, i.e. 2 c_q f*_q for halfway bounce-back.
 *
 * Bounce-back (bb):
 *   0: halfway bounce-back with the true opposite direction;
 *   1: the reference's own table OPP_REF.  For the push kernels (Legacy and
 *      Hybrid) this reproduces the reference's buffer semantics: a slot of
 *      fnext that no thread writes keeps the value the buffer held before
 *      the step (the population of two steps back, after the swap), and a
 *      slot that both a neighbour's streaming and the cell's own bounce-back
 *      write (a race on the GPU in the reference) takes the bounce-back value;
 *   2: as 1, but such a slot takes the streamed value;
 *   3: as 1, but such a slot takes the value of the later loop iteration
 *      (the order within one warp of the reference's kernel).
 */

#define CAT2(a, b) a##b
#define CAT(a, b) CAT2(a, b)
#define FN(name) CAT(name, SUFFIX)

static REAL FN(feq_)(int q, REAL rho, REAL ux, REAL uy, REAL uz) {
    /* src/lbm/lbm3d_legacy.cu:54-58 */
    REAL eiu = (REAL)CX[q] * ux + (REAL)CY[q] * uy + (REAL)CZ[q] * uz;
    REAL uu = ux * ux + uy * uy + uz * uz;
    return WQ(q) * rho * ((REAL)1 + (REAL)3 * eiu + (REAL)4.5 * eiu * eiu - (REAL)1.5 * uu);
}

/* src/lbm/lbm_reinit.cu:20-50 (the cs2 form of the equilibrium) */
void FN(orc_reinit_eq_)(const REAL* rho, const REAL* ux, const REAL* uy, const REAL* uz,
                        REAL* f, int64_t N) {
    const REAL cs2 = (REAL)1 / (REAL)3;
    for (int64_t i = 0; i < N; ++i) {
        const REAL r = rho[i];
        const REAL u0 = ux ? ux[i] : (REAL)0;
        const REAL v0 = uy ? uy[i] : (REAL)0;
        const REAL w0 = uz ? uz[i] : (REAL)0;
        const REAL uu = u0 * u0 + v0 * v0 + w0 * w0;
        for (int q = 0; q < 19; ++q) {
            const REAL cu = (REAL)CX[q] * u0 + (REAL)CY[q] * v0 + (REAL)CZ[q] * w0;
            f[(int64_t)q * N + i] =
                WQ(q) * r * ((REAL)1 + cu / cs2 + (REAL)0.5 * (cu * cu) / (cs2 * cs2) - (REAL)0.5 * uu / cs2);
        }
    }
}

/*
 * One Legacy / Hybrid step, push form, as src/lbm/lbm3d_legacy.cu:59-114 and
 * src/lbm/lbm3d_hybrid.cu:89-175.
 *   mode 0: Legacy BGK everywhere.
 *   mode 1: Hybrid(B0): cells with band[id]!=0 use the BGK form, the others the
 *           "HOME form"  fq + wh(feq-fq) + (ws-wh)(-(fq-feq))  (hybrid.cu:144-153);
 *           band==NULL means no band cells (hybrid.cu:137).
 * Macro outputs are the moments of the incoming f (before collision), with the
 * velocity-shift force added (legacy.cu:78-90,110-113).
 */
void FN(orc_bgk_step_)(const REAL* f, REAL* fn, REAL* rho, REAL* ux, REAL* uy, REAL* uz,
                       const uint8_t* mask, const uint8_t* band, int mode,
                       int nx, int ny, int nz, REAL omega_l, REAL omega_h, REAL omega_s,
                       REAL fx, REAL fy, REAL fz, int bc, REAL u_in, int bb, double* drag) {
    const int64_t N = (int64_t)nx * ny * nz;
    const int* B = bb ? OPP_REF : OPP;
    double dsum[3] = {0, 0, 0};
    /* with true opposites every (q, cell) of fn is written exactly once, so
     * z-rows run in parallel; with the reference's table the streaming writes
     * into a slot that a bounce-back also targets are skipped (bounce wins) */
    #pragma omp parallel for collapse(2) schedule(static) reduction(+:dsum[:3])
    for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
        const int64_t id = ((int64_t)z * ny + y) * nx + x;
        if (mask && mask[id]) {
            for (int q = 0; q < 19; ++q) fn[(int64_t)q * N + id] = f[(int64_t)q * N + id];
            rho[id] = 1; ux[id] = uy[id] = uz[id] = 0;
            continue;
        }
        REAL r = 0, jx = 0, jy = 0, jz = 0;
        for (int q = 0; q < 19; ++q) {
            const REAL fq = f[(int64_t)q * N + id];
            r += fq;
            jx += fq * (REAL)CX[q];
            jy += fq * (REAL)CY[q];
            jz += fq * (REAL)CZ[q];
        }
        REAL u0 = (r > 0) ? jx / r : (REAL)0;
        REAL v0 = (r > 0) ? jy / r : (REAL)0;
        REAL w0 = (r > 0) ? jz / r : (REAL)0;
        u0 += fx; v0 += fy; w0 += fz;
        const int use_bgk = (mode == 0) ? 1 : (band ? (band[id] != 0) : 0);
        REAL fc[19];
        for (int q = 0; q < 19; ++q) {
            const REAL fe = FN(feq_)(q, r, u0, v0, w0);
            const REAL fq = f[(int64_t)q * N + id];
            if (use_bgk) fc[q] = fq + omega_l * (fe - fq);
            else {
                const REAL ds = fq - fe;
                fc[q] = fq + omega_h * (fe - fq) + (omega_s - omega_h) * (-ds);
            }
        }
        for (int q = 0; q < 19; ++q) {
            int x2 = x + CX[q], y2 = y + CY[q], z2 = z + CZ[q];
            y2 = (y2 + ny) % ny; z2 = (z2 + nz) % nz;
            if (bc == 1 && x2 < 0) {               /* inlet link */
                fn[(int64_t)OPP[q] * N + id] = FN(feq_)(OPP[q], r, u_in, 0, 0);
                continue;
            }
            if (bc == 1 && x2 >= nx) {             /* outlet link */
                fn[(int64_t)OPP[q] * N + id] = fc[OPP[q]];
                continue;
            }
            x2 = (x2 + nx) % nx;
            const int64_t id2 = ((int64_t)z2 * ny + y2) * nx + x2;
            if (mask && mask[id2]) {               /* bounce-back into slot B[q] */
                int keep = 1;
                if (bb == 3 && B[q] > q) {
                    /* later loop iteration wins: the streamed write (iteration B[q]) comes after */
                    const int p = B[q];
                    int xs = x - CX[p], ys = (y - CY[p] + ny) % ny, zs = (z - CZ[p] + nz) % nz;
                    if (!(bc == 1 && (xs < 0 || xs >= nx))) {
                        xs = (xs + nx) % nx;
                        keep = mask[((int64_t)zs * ny + ys) * nx + xs] != 0;
                    }
                }
                if (bb == 2) {
                    /* streaming wins: skip when the slot's upstream cell streams into it */
                    const int p = B[q];
                    int xs = x - CX[p], ys = (y - CY[p] + ny) % ny, zs = (z - CZ[p] + nz) % nz;
                    if (!(bc == 1 && (xs < 0 || xs >= nx))) {
                        xs = (xs + nx) % nx;
                        keep = mask[((int64_t)zs * ny + ys) * nx + xs] != 0;
                    }
                }
                if (keep) fn[(int64_t)B[q] * N + id] = fc[q];
                if (!(mask[id2] & 8)) {
                    dsum[0] += (double)(CX[q] - CX[B[q]]) * (double)fc[q];
                    dsum[1] += (double)(CY[q] - CY[B[q]]) * (double)fc[q];
                    dsum[2] += (double)(CZ[q] - CZ[B[q]]) * (double)fc[q];
                }
            } else {
                if ((bb == 1 || (bb == 3 && B[q] > q)) && mask) {
                    /* the target cell's own bounce-back of direction B[q] lands in this slot too */
                    const int p = B[q];
                    int x3 = x2 + CX[p], y3 = (y2 + CY[p] + ny) % ny, z3 = (z2 + CZ[p] + nz) % nz;
                    int skip = 0;
                    if (bc == 1 && (x3 < 0 || x3 >= nx)) skip = 0;
                    else {
                        x3 = (x3 + nx) % nx;
                        skip = mask[((int64_t)z3 * ny + y3) * nx + x3] != 0;
                    }
                    if (skip) continue;
                }
                fn[(int64_t)q * N + id2] = fc[q];
            }
        }
        rho[id] = r; ux[id] = u0; uy[id] = v0; uz[id] = w0;
    }
    if (drag) { drag[0] = dsum[0]; drag[1] = dsum[1]; drag[2] = dsum[2]; }
}

/* src/lbm/lbm3d_home.cu:37-81 */
static REAL FN(rec_post_)(int q, const REAL* c /* rho ux uy uz Sxx Sxy Sxz Syy Syz Szz */,
                          REAL one_minus_omega) {
    const REAL cx = (REAL)CX[q], cy = (REAL)CY[q], cz = (REAL)CZ[q], w = WQ(q);
    const REAL eu = cx * c[1] + cy * c[2] + cz * c[3];
    const REAL uu = c[1] * c[1] + c[2] * c[2] + c[3] * c[3];
    const REAL feq = w * c[0] * ((REAL)1 + (REAL)3 * eu + (REAL)4.5 * eu * eu - (REAL)1.5 * uu);
    const REAL cs2 = (REAL)1 / (REAL)3;
    const REAL Qxx = cx * cx - cs2, Qyy = cy * cy - cs2, Qzz = cz * cz - cs2;
    const REAL Qxy = cx * cy, Qxz = cx * cz, Qyz = cy * cz;
    const REAL con = Qxx * c[4] + Qyy * c[7] + Qzz * c[9] + (REAL)2 * (Qxy * c[5] + Qxz * c[6] + Qyz * c[8]);
    return feq + one_minus_omega * ((REAL)4.5 * w * con);
}

/*
 * One HOME step (moment-only, pull/gather), src/lbm/lbm3d_home.cu:142-286.
 * m / mn hold 10 SoA fields [rho,ux,uy,uz,Sxx,Sxy,Sxz,Syy,Syz,Szz].
 */
void FN(orc_home_step_)(const REAL* m, REAL* mn, const uint8_t* mask,
                        int nx, int ny, int nz, REAL omega, REAL fx, REAL fy, REAL fz,
                        int bc, REAL u_in, int bb, double* drag) {
    const int64_t N = (int64_t)nx * ny * nz;
    const int* B = bb ? OPP_REF : OPP;
    const REAL omw = (REAL)1 - omega;
    double dsum[3] = {0, 0, 0};
    #pragma omp parallel for collapse(2) schedule(static) reduction(+:dsum[:3])
    for (int z = 0; z < nz; ++z)
    for (int y = 0; y < ny; ++y)
    for (int x = 0; x < nx; ++x) {
        const int64_t id = ((int64_t)z * ny + y) * nx + x;
        if (mask && mask[id]) {
            mn[id] = 1;
            for (int k = 1; k < 10; ++k) mn[(int64_t)k * N + id] = 0;
            continue;
        }
        REAL own[10];
        for (int k = 0; k < 10; ++k) own[k] = m[(int64_t)k * N + id];
        REAL r = 0, jx = 0, jy = 0, jz = 0, Mxx = 0, Mxy = 0, Mxz = 0, Myy = 0, Myz = 0, Mzz = 0;
        for (int q = 0; q < 19; ++q) {
            int xs = x - CX[q], ys = y - CY[q], zs = z - CZ[q];
            ys = (ys + ny) % ny; zs = (zs + nz) % nz;
            REAL fq;
            if (bc == 1 && xs < 0) {
                fq = FN(feq_)(q, own[0], u_in, 0, 0);
            } else if (bc == 1 && xs >= nx) {
                fq = FN(rec_post_)(q, own, omw);
            } else {
                xs = (xs + nx) % nx;
                const int64_t ids = ((int64_t)zs * ny + ys) * nx + xs;
                if (mask && mask[ids]) {
                    /* the own post-collision population of direction B[q] comes back as q
                     * (home.cu:219-225) */
                    fq = FN(rec_post_)(B[q], own, omw);
                    if (!(mask[ids] & 8)) {
                        dsum[0] += (double)(CX[B[q]] - CX[q]) * (double)fq;
                        dsum[1] += (double)(CY[B[q]] - CY[q]) * (double)fq;
                        dsum[2] += (double)(CZ[B[q]] - CZ[q]) * (double)fq;
                    }
                } else {
                    REAL nb[10];
                    for (int k = 0; k < 10; ++k) nb[k] = m[(int64_t)k * N + ids];
                    fq = FN(rec_post_)(q, nb, omw);
                }
            }
            const REAL cx = (REAL)CX[q], cy = (REAL)CY[q], cz = (REAL)CZ[q];
            r += fq; jx += fq * cx; jy += fq * cy; jz += fq * cz;
            Mxx += fq * cx * cx; Mxy += fq * cx * cy; Mxz += fq * cx * cz;
            Myy += fq * cy * cy; Myz += fq * cy * cz; Mzz += fq * cz * cz;
        }
        REAL u = (r > 0) ? jx / r : (REAL)0;
        REAL v = (r > 0) ? jy / r : (REAL)0;
        REAL w = (r > 0) ? jz / r : (REAL)0;
        u += fx; v += fy; w += fz;
        const REAL cs2 = (REAL)1 / (REAL)3;
        mn[id] = r;
        mn[1 * N + id] = u;
        mn[2 * N + id] = v;
        mn[3 * N + id] = w;
        mn[4 * N + id] = Mxx - (r * cs2 + r * u * u);
        mn[5 * N + id] = Mxy - r * u * v;
        mn[6 * N + id] = Mxz - r * u * w;
        mn[7 * N + id] = Myy - (r * cs2 + r * v * v);
        mn[8 * N + id] = Myz - r * v * w;
        mn[9 * N + id] = Mzz - (r * cs2 + r * w * w);
    }
    if (drag) { drag[0] = dsum[0]; drag[1] = dsum[1]; drag[2] = dsum[2]; }
}

/* Run n steps with ping-pong buffers; the final state is left in a and the other
 * buffer in b, as after the reference's swap (src/lbm/lbm3d_legacy.cu:115-118,218-220):
 * b must hold what the reference's fnext holds on entry (a copy of f after
 * reinitEquilibriumFromMacro, legacy.cu:205-206). */
void FN(orc_bgk_run_)(REAL* a, REAL* b, REAL* rho, REAL* ux, REAL* uy, REAL* uz,
                      const uint8_t* mask, const uint8_t* band, int mode,
                      int nx, int ny, int nz, REAL omega_l, REAL omega_h, REAL omega_s,
                      REAL fx, REAL fy, REAL fz, int bc, REAL u_in, int bb, int nsteps, double* drag) {
    const int64_t n19 = (int64_t)19 * nx * ny * nz;
    REAL *cur = a, *nxt = b;
    for (int s = 0; s < nsteps; ++s) {
        FN(orc_bgk_step_)(cur, nxt, rho, ux, uy, uz, mask, band, mode, nx, ny, nz,
                          omega_l, omega_h, omega_s, fx, fy, fz, bc, u_in, bb, drag);
        REAL* t = cur; cur = nxt; nxt = t;
    }
    if (cur != a) {   /* odd count: exchange the two buffers' contents */
        REAL* t = (REAL*)malloc(sizeof(REAL) * (size_t)n19);
        memcpy(t, a, sizeof(REAL) * (size_t)n19);
        memcpy(a, cur, sizeof(REAL) * (size_t)n19);
        memcpy(b, t, sizeof(REAL) * (size_t)n19);
        free(t);
    }
}

void FN(orc_home_run_)(REAL* a, REAL* b, const uint8_t* mask, int nx, int ny, int nz,
                       REAL omega, REAL fx, REAL fy, REAL fz, int bc, REAL u_in, int bb, int nsteps,
                       double* drag) {
    const int64_t n10 = (int64_t)10 * nx * ny * nz;
    REAL *cur = a, *nxt = b;
    for (int s = 0; s < nsteps; ++s) {
        FN(orc_home_step_)(cur, nxt, mask, nx, ny, nz, omega, fx, fy, fz, bc, u_in, bb, drag);
        REAL* t = cur; cur = nxt; nxt = t;
    }
    if (cur != a) memcpy(a, cur, sizeof(REAL) * (size_t)n10);
}

#undef FN
