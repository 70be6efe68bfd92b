/*
 * plate_oracle.c -- CPU restatement of the reference plate solver.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the checker for the CUDA solver:
 * only tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg load
 * it.  Nothing in the product links or calls it.
 *
 * It restates, in C, the reference's CPU solver for the matrix-free
 * plate-bending PCG path of cseifert512/gpu-gauntlet (TypeScript):
 *   src/lib/plate/element.ts   Q4 Mindlin Ke (:258-483) and DKT Ke (:642-943)
 *   src/lib/plate/solver.ts    supports (:92-134), diagonal (:145-177),
 *                              block diagonal + inversion (:188-304),
 *                              block preconditioner (:313-339),
 *                              loads / RHS BCs (:363-407), K.x (:422-483)
 *   src/lib/plate/pcg.ts       solvePCG (:98-215), solveTestSystem (:221-247)
 *   src/lib/plate/coloring.ts  structured (:38-81), greedy (:92-177),
 *                              verifyColoring (:188-225)
 *   src/lib/plate/mesher.ts    generateRectangularMesh (:364-439)
 *
 * Two arithmetic modes:
 *   OR_REF  (0): reference precision.  Every value the reference keeps in a
 *                Float32Array (Ke, Db/Ds, B/DB, block diagonal, vectors x, r,
 *                z, p, Ap, y, F) is rounded to binary32 on every store, and
 *                every intermediate is a binary64 JS number.  Compiled with
 *                -ffp-contract=off so that a*b+c is never fused (JS never
 *                fuses), which makes this mode reproduce the JS arithmetic
 *                operation for operation.  pow() comes from the C library
 *                (V8 uses an fdlibm port; the two agree to <= 1 ulp).
 *   OR_FP64 (1): the same formulas with no binary32 rounding at all (node
 *                coordinates stay the binary32 values the mesh holds).  This
 *                is the operator the GPU solver applies and the FP64 truth.
 *
 * Parity pinning: the reference ships no tests, fixtures or recorded
 * outputs and its JavaScript cannot run in this image (no Node).  The
 * restatement is pinned by the reference's own known-answer system
 * (solveTestSystem, pcg.ts:221-247, x = ones(10)), by verifyColoring, by the
 * element checks isSymmetric / isPositiveSemiDefinite (element.ts:568-597),
 * and by external physics (Kirchhoff plate coefficients).  Element-level
 * values are otherwise "parity partially pinned": pinned by restated code,
 * not by outputs recorded from the reference.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define OR_REF 0
#define OR_FP64 1

/* Store rounding: a Float32Array store in OR_REF mode (Math.fround). */
static inline double R(int mode, double v) { return mode == OR_REF ? (double)(float)v : v; }

/* types.ts:26-28 */
static double flexural_rigidity(double E, double nu, double t) {
    return (E * pow(t, 3.0)) / (12.0 * (1.0 - pow(nu, 2.0)));
}

/* ------------------------------------------------------------------------ */
/* element.ts: Q4 Mindlin                                                   */
/* ------------------------------------------------------------------------ */

static const double GP_2X2 = 0.5773502691896257; /* element.ts:30 */

/* element.ts:80-106 */
static void shape_derivs(double xi, double eta, double dNdXi[4], double dNdEta[4]) {
    double xm = 1 - xi, xp = 1 + xi, em = 1 - eta, ep = 1 + eta;
    dNdXi[0] = -em / 4; dNdXi[1] = +em / 4; dNdXi[2] = +ep / 4; dNdXi[3] = -ep / 4;
    dNdEta[0] = -xm / 4; dNdEta[1] = -xp / 4; dNdEta[2] = +xp / 4; dNdEta[3] = +xm / 4;
}

/* element.ts:119-148 and :162-184 */
static double phys_derivs(const float *c, const double dNdXi[4], const double dNdEta[4],
                          double dNdx[4], double dNdy[4]) {
    double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
    for (int i = 0; i < 4; i++) {
        double x = c[i * 2], y = c[i * 2 + 1];
        J11 += dNdXi[i] * x;
        J12 += dNdXi[i] * y;
        J21 += dNdEta[i] * x;
        J22 += dNdEta[i] * y;
    }
    double detJ = J11 * J22 - J12 * J21;
    double invDetJ = 1.0 / detJ;
    for (int i = 0; i < 4; i++) {
        dNdx[i] = invDetJ * (J22 * dNdXi[i] - J12 * dNdEta[i]);
        dNdy[i] = invDetJ * (-J21 * dNdXi[i] + J11 * dNdEta[i]);
    }
    return detJ;
}

/* computeElementStiffness, element.ts:258-483.  Ke row-major 12x12. */
void or_q4_ke(const float *coords, double E, double nu, double t, int mode, double *Ke) {
    for (int i = 0; i < 144; i++) Ke[i] = 0.0;
    double D = flexural_rigidity(E, nu, t);
    /* Db / Ds are Float32Array in the reference (element.ts:209-219, :239) */
    double D11 = R(mode, D), D12 = R(mode, D * nu), D22 = R(mode, D);
    double D33 = R(mode, (D * (1 - nu)) / 2);
    double kappa = 5.0 / 6.0;
    double G = E / (2 * (1 + nu));
    double Dsc = R(mode, kappa * G * t);
    double Ds11 = Dsc, Ds22 = Dsc;

    static const double pts[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    for (int gp = 0; gp < 4; gp++) {
        double xi = pts[gp][0] * GP_2X2, eta = pts[gp][1] * GP_2X2;
        double weight = 1.0;
        double dNdXi[4], dNdEta[4], dNdx[4], dNdy[4];
        shape_derivs(xi, eta, dNdXi, dNdEta);
        double detJ = phys_derivs(coords, dNdXi, dNdEta, dNdx, dNdy);
        double factor = weight * fabs(detJ);
        for (int i = 0; i < 4; i++) {
            for (int j = 0; j < 4; j++) {
                int di_tx = i * 3 + 1, di_ty = i * 3 + 2, dj_tx = j * 3 + 1, dj_ty = j * 3 + 2;
                double dNdx_i = dNdx[i], dNdy_i = dNdy[i], dNdx_j = dNdx[j], dNdy_j = dNdy[j];
                double K_tx_tx = dNdy_i * D22 * dNdy_j + dNdx_i * D33 * dNdx_j;
                double K_ty_ty = dNdx_i * D11 * dNdx_j + dNdy_i * D33 * dNdy_j;
                double K_tx_ty = -dNdy_i * D12 * dNdx_j - dNdx_i * D33 * dNdy_j;
                double K_ty_tx = -dNdx_i * D12 * dNdy_j - dNdy_i * D33 * dNdx_j;
                Ke[di_tx * 12 + dj_tx] = R(mode, Ke[di_tx * 12 + dj_tx] + factor * K_tx_tx);
                Ke[di_ty * 12 + dj_ty] = R(mode, Ke[di_ty * 12 + dj_ty] + factor * K_ty_ty);
                Ke[di_tx * 12 + dj_ty] = R(mode, Ke[di_tx * 12 + dj_ty] + factor * K_tx_ty);
                Ke[di_ty * 12 + dj_tx] = R(mode, Ke[di_ty * 12 + dj_tx] + factor * K_ty_tx);
            }
        }
    }
    {
        /* shear, 1-point rule at the centre, weight 4 (element.ts:390-480) */
        double xi = 0, eta = 0, weight = 4.0;
        double xm = 1 - xi, xp = 1 + xi, em = 1 - eta, ep = 1 + eta;
        double N[4] = {(xm * em) / 4, (xp * em) / 4, (xp * ep) / 4, (xm * ep) / 4};
        double dNdXi[4], dNdEta[4], dNdx[4], dNdy[4];
        shape_derivs(xi, eta, dNdXi, dNdEta);
        double detJ = phys_derivs(coords, dNdXi, dNdEta, dNdx, dNdy);
        double factor = weight * fabs(detJ);
        for (int i = 0; i < 4; i++) {
            for (int j = 0; j < 4; j++) {
                int di_w = i * 3, di_tx = i * 3 + 1, di_ty = i * 3 + 2;
                int dj_w = j * 3, dj_tx = j * 3 + 1, dj_ty = j * 3 + 2;
                double N_i = N[i], N_j = N[j];
                double dNdx_i = dNdx[i], dNdy_i = dNdy[i], dNdx_j = dNdx[j], dNdy_j = dNdy[j];
                double K_w_w = dNdx_i * Ds11 * dNdx_j + dNdy_i * Ds22 * dNdy_j;
                double K_w_tx = dNdy_i * Ds22 * (-N_j);
                double K_w_ty = dNdx_i * Ds11 * N_j;
                double K_tx_w = (-N_i) * Ds22 * dNdy_j;
                double K_tx_tx = (-N_i) * Ds22 * (-N_j);
                double K_ty_w = N_i * Ds11 * dNdx_j;
                double K_ty_ty = N_i * Ds11 * N_j;
                Ke[di_w * 12 + dj_w] = R(mode, Ke[di_w * 12 + dj_w] + factor * K_w_w);
                Ke[di_w * 12 + dj_tx] = R(mode, Ke[di_w * 12 + dj_tx] + factor * K_w_tx);
                Ke[di_w * 12 + dj_ty] = R(mode, Ke[di_w * 12 + dj_ty] + factor * K_w_ty);
                Ke[di_tx * 12 + dj_w] = R(mode, Ke[di_tx * 12 + dj_w] + factor * K_tx_w);
                Ke[di_tx * 12 + dj_tx] = R(mode, Ke[di_tx * 12 + dj_tx] + factor * K_tx_tx);
                /* K_tx_ty and K_ty_tx are 0: adding factor*0 leaves the entry unchanged */
                Ke[di_ty * 12 + dj_w] = R(mode, Ke[di_ty * 12 + dj_w] + factor * K_ty_w);
                Ke[di_ty * 12 + dj_ty] = R(mode, Ke[di_ty * 12 + dj_ty] + factor * K_ty_ty);
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* element.ts: DKT                                                          */
/* ------------------------------------------------------------------------ */

/* computeDKTBx, element.ts:833-887 */
static void dkt_bx(int mode, double L1, double L2, double P4, double P5, double P6, double q4,
                   double q5, double q6, double c4, double c5, double c6, double d1[9], double d2[9]) {
    d1[0] = R(mode, P6 * (1 - 2 * L1) + (P5 - P6) * L2);
    d1[1] = R(mode, q6 * (1 - 2 * L1) - (q5 + q6) * L2);
    d1[2] = R(mode, -4 + 6 * (L1 + L2) + (c5 - c6) * L2 + c6 * (1 - 2 * L1));
    d2[0] = R(mode, -P6 * (1 - 2 * L2) + (P4 - P5) * L1 - P5 * (1 - 2 * L2));
    d2[1] = R(mode, q6 * (1 - 2 * L2) - (q4 + q5) * L1 + q5 * (1 - 2 * L2));
    d2[2] = R(mode, -4 + 6 * (L1 + L2) + (c4 - c5) * L1 + c5 * (1 - 2 * L2));
    d1[3] = R(mode, P4 * L2 + P6 * (1 - 2 * L1));
    d1[4] = R(mode, q4 * L2 - q6 * (1 - 2 * L1));
    d1[5] = R(mode, c4 * L2 - c6 * (1 - 2 * L1));
    d2[3] = R(mode, P4 * (1 - 2 * L2) + P5 * L1);
    d2[4] = R(mode, q4 * (1 - 2 * L2) - q5 * L1);
    d2[5] = R(mode, c4 * (1 - 2 * L2) - c5 * L1);
    d1[6] = R(mode, -P5 * L2 - P6 * (1 - 2 * L1));
    d1[7] = R(mode, q5 * L2 + q6 * (1 - 2 * L1));
    d1[8] = R(mode, -c5 * L2 + c6 * (1 - 2 * L1));
    d2[6] = R(mode, -P4 * L1 - P5 * (1 - 2 * L2));
    d2[7] = R(mode, q4 * L1 + q5 * (1 - 2 * L2));
    d2[8] = R(mode, -c4 * L1 + c5 * (1 - 2 * L2));
}

/* computeDKTBy, element.ts:893-943 */
static void dkt_by(int mode, double L1, double L2, double t4, double t5, double t6, double r4,
                   double r5, double r6, double e4, double e5, double e6, double b4, double b5,
                   double b6, double d1[9], double d2[9]) {
    (void)b4;
    d1[0] = R(mode, t6 * (1 - 2 * L1) + (t5 - t6) * L2);
    d1[1] = R(mode, 1 + r6 * (1 - 2 * L1) - (r5 + r6) * L2);
    d1[2] = R(mode, -e6 * (1 - 2 * L1) + (b5 - b6) * L2);
    d2[0] = R(mode, -t6 * (1 - 2 * L2) + (t4 - t5) * L1 - t5 * (1 - 2 * L2));
    d2[1] = R(mode, 1 + r6 * (1 - 2 * L2) - (r4 + r5) * L1 + r5 * (1 - 2 * L2));
    d2[2] = R(mode, e6 * (1 - 2 * L2) + (b4 - b5) * L1 - b5 * (1 - 2 * L2));
    d1[3] = R(mode, t4 * L2 + t6 * (1 - 2 * L1));
    d1[4] = R(mode, -1 + r4 * L2 - r6 * (1 - 2 * L1));
    d1[5] = R(mode, -e4 * L2 - b6 * (1 - 2 * L1));
    d2[3] = R(mode, t4 * (1 - 2 * L2) + t5 * L1);
    d2[4] = R(mode, -1 + r4 * (1 - 2 * L2) - r5 * L1);
    d2[5] = R(mode, -e4 * (1 - 2 * L2) + b5 * L1);
    d1[6] = R(mode, -t5 * L2 - t6 * (1 - 2 * L1));
    d1[7] = R(mode, r5 * L2 + r6 * (1 - 2 * L1));
    d1[8] = R(mode, e5 * L2 + b6 * (1 - 2 * L1));
    d2[6] = R(mode, -t4 * L1 - t5 * (1 - 2 * L2));
    d2[7] = R(mode, r4 * L1 + r5 * (1 - 2 * L2));
    d2[8] = R(mode, e4 * L1 - b5 * (1 - 2 * L2));
}

/* computeDKTStiffness, element.ts:642-827.  Ke row-major 9x9. */
void or_dkt_ke(const float *c, double E, double nu, double t, int mode, double *Ke) {
    for (int i = 0; i < 81; i++) Ke[i] = 0.0;
    double x1 = c[0], y1 = c[1], x2 = c[2], y2 = c[3], x3 = c[4], y3 = c[5];
    double x12 = x1 - x2, y12 = y1 - y2;
    double x23 = x2 - x3, y23 = y2 - y3;
    double x31 = x3 - x1, y31 = y3 - y1;
    double L12_sq = x12 * x12 + y12 * y12;
    double L23_sq = x23 * x23 + y23 * y23;
    double L31_sq = x31 * x31 + y31 * y31;
    double twoA = x12 * y31 - x31 * y12;
    double area = fabs(twoA) / 2;
    if (area < 1e-15) return; /* degenerate: zero Ke (element.ts:672-676) */

    double D = flexural_rigidity(E, nu, t);
    double D11 = D, D12 = D * nu, D22 = D, D33 = (D * (1 - nu)) / 2;

    double a4 = -x23 / L23_sq, b4 = (3 * x23 * y23) / (4 * L23_sq);
    double c4 = (x23 * x23 - 2 * y23 * y23) / (4 * L23_sq), d4 = -y23 / L23_sq;
    double e4 = (y23 * y23 - 2 * x23 * x23) / (4 * L23_sq);
    double a5 = -x31 / L31_sq, b5 = (3 * x31 * y31) / (4 * L31_sq);
    double c5 = (x31 * x31 - 2 * y31 * y31) / (4 * L31_sq), d5 = -y31 / L31_sq;
    double e5 = (y31 * y31 - 2 * x31 * x31) / (4 * L31_sq);
    double a6 = -x12 / L12_sq, b6 = (3 * x12 * y12) / (4 * L12_sq);
    double c6 = (x12 * x12 - 2 * y12 * y12) / (4 * L12_sq), d6 = -y12 / L12_sq;
    double e6 = (y12 * y12 - 2 * x12 * x12) / (4 * L12_sq);
    double P4 = -6 * a4, P5 = -6 * a5, P6 = -6 * a6;
    double t4 = -6 * d4, t5 = -6 * d5, t6 = -6 * d6;
    double q4 = 3 * a4, q5 = 3 * a5, q6 = 3 * a6;
    double r4 = 3 * d4, r5 = 3 * d5, r6 = 3 * d6;

    static const double gpts[3][3] = {
        {1.0 / 6, 1.0 / 6, 2.0 / 3}, {2.0 / 3, 1.0 / 6, 1.0 / 6}, {1.0 / 6, 2.0 / 3, 1.0 / 6}};
    for (int gp = 0; gp < 3; gp++) {
        double L1 = gpts[gp][0], L2 = gpts[gp][1];
        double weight = 1.0 / 3;
        double bx1[9], bx2[9], by1[9], by2[9];
        dkt_bx(mode, L1, L2, P4, P5, P6, q4, q5, q6, c4, c5, c6, bx1, bx2);
        dkt_by(mode, L1, L2, t4, t5, t6, r4, r5, r6, e4, e5, e6, b4, b5, b6, by1, by2);
        double invTwoA = 1 / twoA;
        double B[27], DB[27];
        for (int j = 0; j < 9; j++) {
            B[0 * 9 + j] = R(mode, invTwoA * ((-y23) * bx1[j] + (-y31) * bx2[j]));
            B[1 * 9 + j] = R(mode, invTwoA * (x23 * by1[j] + x31 * by2[j]));
            B[2 * 9 + j] = R(mode, invTwoA * (x23 * bx1[j] + x31 * bx2[j] + (-y23) * by1[j] +
                                              (-y31) * by2[j]));
        }
        double factor = weight * area;
        for (int j = 0; j < 9; j++) {
            DB[0 * 9 + j] = R(mode, D11 * B[0 * 9 + j] + D12 * B[1 * 9 + j]);
            DB[1 * 9 + j] = R(mode, D12 * B[0 * 9 + j] + D22 * B[1 * 9 + j]);
            DB[2 * 9 + j] = R(mode, D33 * B[2 * 9 + j]);
        }
        for (int i = 0; i < 9; i++) {
            for (int j = 0; j < 9; j++) {
                double sum = 0;
                for (int k = 0; k < 3; k++) sum += B[k * 9 + i] * DB[k * 9 + j];
                Ke[i * 9 + j] = R(mode, Ke[i * 9 + j] + factor * sum);
            }
        }
    }
}

/* ------------------------------------------------------------------------ */
/* mesher.ts:364-439 generateRectangularMesh                                 */
/* ------------------------------------------------------------------------ */

void or_rect_dims(double width, double height, double target, int *nx, int *ny) {
    double cx = ceil(width / target), cy = ceil(height / target);
    *nx = (int)(cx > 2 ? cx : 2);
    *ny = (int)(cy > 2 ? cy : 2);
}

/* nodes: 2*(nx+1)*(ny+1) floats, elements: 4*nx*ny, boundary: 2*(nx+ny) */
void or_rect_mesh(double width, double height, int nx, int ny, float *nodes, uint32_t *elements,
                  uint32_t *boundary) {
    double dx = width / nx, dy = height / ny;
    int nodesX = nx + 1;
    for (int j = 0; j <= ny; j++)
        for (int i = 0; i <= nx; i++) {
            int idx = j * nodesX + i;
            nodes[idx * 2] = (float)(i * dx);
            nodes[idx * 2 + 1] = (float)(j * dy);
        }
    int e = 0;
    for (int j = 0; j < ny; j++)
        for (int i = 0; i < nx; i++) {
            elements[e * 4 + 0] = j * nodesX + i;
            elements[e * 4 + 1] = j * nodesX + (i + 1);
            elements[e * 4 + 2] = (j + 1) * nodesX + (i + 1);
            elements[e * 4 + 3] = (j + 1) * nodesX + i;
            e++;
        }
    int b = 0;
    for (int i = 0; i <= nx; i++) boundary[b++] = i;
    for (int j = 1; j <= ny; j++) boundary[b++] = j * nodesX + nx;
    for (int i = nx - 1; i >= 0; i--) boundary[b++] = ny * nodesX + i;
    for (int j = ny - 1; j >= 1; j--) boundary[b++] = j * nodesX;
}

/* ------------------------------------------------------------------------ */
/* coloring.ts                                                              */
/* ------------------------------------------------------------------------ */

/* computeElementColoring, coloring.ts:38-81.  colors_flat holds the colour
 * lists back to back (colour 0 first); counts[4]. */
void or_color_structured(int Ne, int gridNx, uint8_t *elementColors, uint32_t *colors_flat,
                         int *counts) {
    for (int c = 0; c < 4; c++) counts[c] = 0;
    for (int e = 0; e < Ne; e++) {
        int i = e % gridNx, j = e / gridNx;
        int color = (i % 2) * 2 + (j % 2);
        elementColors[e] = (uint8_t)color;
        counts[color]++;
    }
    int off[4] = {0, counts[0], counts[0] + counts[1], counts[0] + counts[1] + counts[2]};
    for (int e = 0; e < Ne; e++) colors_flat[off[elementColors[e]]++] = (uint32_t)e;
}

/* node -> elements CSR (element ids ascending per node) */
static void node_elems(int Nn, int Ne, int npe, const uint32_t *el, int **ptr_out, int **idx_out) {
    int *ptr = (int *)calloc((size_t)Nn + 1, sizeof(int));
    for (int e = 0; e < Ne; e++)
        for (int k = 0; k < npe; k++) ptr[el[e * npe + k] + 1]++;
    for (int n = 0; n < Nn; n++) ptr[n + 1] += ptr[n];
    int *idx = (int *)malloc(sizeof(int) * (size_t)(ptr[Nn] > 0 ? ptr[Nn] : 1));
    int *fill = (int *)malloc(sizeof(int) * (size_t)(Nn > 0 ? Nn : 1));
    for (int n = 0; n < Nn; n++) fill[n] = ptr[n];
    for (int e = 0; e < Ne; e++)
        for (int k = 0; k < npe; k++) idx[fill[el[e * npe + k]]++] = e;
    free(fill);
    *ptr_out = ptr;
    *idx_out = idx;
}

/* computeElementColoringGreedy, coloring.ts:92-177.  Returns colorCount;
 * counts must hold up to 256 entries. */
int or_color_greedy(int Nn, int Ne, int npe, const uint32_t *el, uint8_t *elementColors,
                    uint32_t *colors_flat, int *counts) {
    int *ptr, *idx;
    node_elems(Nn, Ne, npe, el, &ptr, &idx);
    for (int e = 0; e < Ne; e++) elementColors[e] = 255;
    int maxColor = 0;
    int used[257];
    for (int e = 0; e < Ne; e++) {
        memset(used, 0, sizeof(used));
        for (int k = 0; k < npe; k++) {
            int n = (int)el[e * npe + k];
            for (int q = ptr[n]; q < ptr[n + 1]; q++) {
                int nb = idx[q];
                if (nb != e && elementColors[nb] != 255) used[elementColors[nb]] = 1;
            }
        }
        int color = 0;
        while (used[color]) color++;
        elementColors[e] = (uint8_t)color;
        if (color > maxColor) maxColor = color;
    }
    int colorCount = Ne > 0 ? maxColor + 1 : 1;
    for (int c = 0; c < colorCount; c++) counts[c] = 0;
    for (int e = 0; e < Ne; e++) counts[elementColors[e]]++;
    int off[256];
    int acc = 0;
    for (int c = 0; c < colorCount; c++) { off[c] = acc; acc += counts[c]; }
    for (int e = 0; e < Ne; e++) colors_flat[off[elementColors[e]]++] = (uint32_t)e;
    free(ptr);
    free(idx);
    return colorCount;
}

/* verifyColoring, coloring.ts:188-225.  1 = valid. */
int or_verify_coloring(int Nn, int Ne, int npe, const uint32_t *el, const uint8_t *elementColors) {
    int *ptr, *idx;
    node_elems(Nn, Ne, npe, el, &ptr, &idx);
    int ok = 1;
    for (int n = 0; n < Nn && ok; n++) {
        int seen[256] = {0};
        for (int q = ptr[n]; q < ptr[n + 1]; q++) {
            int c = elementColors[idx[q]];
            if (seen[c]) { ok = 0; break; }
            seen[c] = 1;
        }
    }
    free(ptr);
    free(idx);
    return ok;
}

/* ------------------------------------------------------------------------ */
/* solver.ts                                                                */
/* ------------------------------------------------------------------------ */

/* Ke of every element (the reference's Ke cache, solver.ts:49-77).
 * ke_all: Ne * (3*npe)^2 doubles.  elem_t (nullable) overrides the
 * thickness per element (an extension; the reference has a scalar t). */
void or_all_ke(int Ne, int npe, const float *nodes, const uint32_t *el, double E, double nu,
               double t, const float *elem_t, int mode, double *ke_all) {
    int nd = 3 * npe, kk = nd * nd;
    for (int e = 0; e < Ne; e++) {
        float c[8];
        for (int k = 0; k < npe; k++) {
            uint32_t n = el[e * npe + k];
            c[k * 2] = nodes[n * 2];
            c[k * 2 + 1] = nodes[n * 2 + 1];
        }
        double te = elem_t ? (double)elem_t[e] : t;
        if (npe == 3)
            or_dkt_ke(c, E, nu, te, mode, ke_all + (size_t)e * kk);
        else
            or_q4_ke(c, E, nu, te, mode, ke_all + (size_t)e * kk);
    }
}

/* computeDiagonal, solver.ts:145-177 (element order, += per store) */
void or_diagonal(int Nn, int Ne, int npe, const uint32_t *el, const double *ke_all, int mode,
                 double *diag) {
    int nd = 3 * npe, kk = nd * nd;
    for (int i = 0; i < Nn * 3; i++) diag[i] = 0.0;
    for (int e = 0; e < Ne; e++) {
        const double *Ke = ke_all + (size_t)e * kk;
        for (int i = 0; i < npe; i++) {
            uint32_t g = el[e * npe + i];
            for (int d = 0; d < 3; d++) {
                int l = i * 3 + d;
                diag[g * 3 + d] = R(mode, diag[g * 3 + d] + Ke[l * nd + l]);
            }
        }
    }
}

/* computeBlockDiagonal, solver.ts:188-225 */
void or_block_diag(int Nn, int Ne, int npe, const uint32_t *el, const double *ke_all, int mode,
                   double *bd) {
    int nd = 3 * npe, kk = nd * nd;
    for (int i = 0; i < Nn * 9; i++) bd[i] = 0.0;
    for (int e = 0; e < Ne; e++) {
        const double *Ke = ke_all + (size_t)e * kk;
        for (int i = 0; i < npe; i++) {
            uint32_t g = el[e * npe + i];
            int lb = i * 3;
            for (int r = 0; r < 3; r++)
                for (int c = 0; c < 3; c++) {
                    double *dst = &bd[g * 9 + r * 3 + c];
                    *dst = R(mode, *dst + Ke[(lb + r) * nd + lb + c]);
                }
        }
    }
}

/* invertBlockDiagonal, solver.ts:231-304 (in place) */
void or_invert_block_diag(int Nn, double *bd, const uint8_t *cons, int mode) {
    for (int node = 0; node < Nn; node++) {
        double *b = bd + node * 9;
        int wc = cons[node * 3], txc = cons[node * 3 + 1], tyc = cons[node * 3 + 2];
        if (wc && txc && tyc) {
            for (int k = 0; k < 9; k++) b[k] = (k % 4 == 0) ? 1.0 : 0.0;
            continue;
        }
        if (wc) { b[0] = 1; b[1] = 0; b[2] = 0; b[3] = 0; b[6] = 0; }
        if (txc) { b[4] = 1; b[1] = 0; b[7] = 0; b[3] = 0; b[5] = 0; }
        if (tyc) { b[8] = 1; b[2] = 0; b[5] = 0; b[6] = 0; b[7] = 0; }
        double a00 = b[0], a01 = b[1], a02 = b[2];
        double a10 = b[3], a11 = b[4], a12 = b[5];
        double a20 = b[6], a21 = b[7], a22 = b[8];
        double det = a00 * (a11 * a22 - a12 * a21) - a01 * (a10 * a22 - a12 * a20) +
                     a02 * (a10 * a21 - a11 * a20);
        if (fabs(det) < 1e-30) {
            for (int k = 0; k < 9; k++) b[k] = (k % 4 == 0) ? 1.0 : 0.0;
            continue;
        }
        double invDet = 1.0 / det;
        b[0] = R(mode, invDet * (a11 * a22 - a12 * a21));
        b[1] = R(mode, invDet * (a02 * a21 - a01 * a22));
        b[2] = R(mode, invDet * (a01 * a12 - a02 * a11));
        b[3] = R(mode, invDet * (a12 * a20 - a10 * a22));
        b[4] = R(mode, invDet * (a00 * a22 - a02 * a20));
        b[5] = R(mode, invDet * (a02 * a10 - a00 * a12));
        b[6] = R(mode, invDet * (a10 * a21 - a11 * a20));
        b[7] = R(mode, invDet * (a01 * a20 - a00 * a21));
        b[8] = R(mode, invDet * (a00 * a11 - a01 * a10));
    }
}

/* applyBlockPreconditioner, solver.ts:313-339 / pcg.ts:74-88 */
void or_block_precond(int Nn, const double *bi, const double *r, double *z, int mode) {
    for (int node = 0; node < Nn; node++) {
        const double *b = bi + node * 9;
        double r0 = r[node * 3], r1 = r[node * 3 + 1], r2 = r[node * 3 + 2];
        z[node * 3] = R(mode, b[0] * r0 + b[1] * r1 + b[2] * r2);
        z[node * 3 + 1] = R(mode, b[3] * r0 + b[4] * r1 + b[5] * r2);
        z[node * 3 + 2] = R(mode, b[6] * r0 + b[7] * r1 + b[8] * r2);
    }
}

/* identifyConstrainedDOFs, solver.ts:92-134.  support types: 0 pinned,
 * 1 fixed, 2 roller; location < 0 means 'all_edges'.  cons is OR-ed. */
void or_constrained(int nsup, const int *types, const int *locations, int nboundary,
                    const uint32_t *boundary, uint8_t *cons) {
    for (int s = 0; s < nsup; s++) {
        int count = locations[s] < 0 ? nboundary : 1;
        for (int q = 0; q < count; q++) {
            int node = locations[s] < 0 ? (int)boundary[q] : locations[s];
            cons[node * 3] = 1;
            if (types[s] == 1) { cons[node * 3 + 1] = 1; cons[node * 3 + 2] = 1; }
        }
    }
}

/* buildLoadVector, solver.ts:363-392 (nearest node, first minimum wins) */
void or_load_vector(int Nn, const float *nodes, int nloads, const double *pos, const double *mag,
                    int mode, double *F) {
    for (int i = 0; i < Nn * 3; i++) F[i] = 0.0;
    for (int l = 0; l < nloads; l++) {
        double px = pos[2 * l], py = pos[2 * l + 1];
        int nearest = 0;
        double minDist = INFINITY;
        for (int i = 0; i < Nn; i++) {
            double nx = nodes[i * 2], ny = nodes[i * 2 + 1];
            double dist = sqrt((nx - px) * (nx - px) + (ny - py) * (ny - py));
            if (dist < minDist) { minDist = dist; nearest = i; }
        }
        F[nearest * 3] = R(mode, F[nearest * 3] + mag[l]);
    }
}

/* applyBCsToRHS, solver.ts:400-407 */
void or_apply_bcs_rhs(int n, const uint8_t *cons, double *F) {
    for (int i = 0; i < n; i++)
        if (cons[i]) F[i] = 0.0;
}

/* applyGlobalK, solver.ts:422-483.  Colours in order, elements in colour-list
 * order, each yLocal row rounded then added into y; constrained rows copy x. */
void or_apply_k(int Nn, int npe, const uint32_t *el, const double *ke_all, int ncolors,
                const int *color_offsets, const uint32_t *elements_by_color, const uint8_t *cons,
                const double *x, double *y, int mode) {
    int nd = 3 * npe, kk = nd * nd;
    for (int i = 0; i < Nn * 3; i++) y[i] = 0.0;
    int dofs[12];
    double xl[12], yl[12];
    for (int c = 0; c < ncolors; c++) {
        for (int q = color_offsets[c]; q < color_offsets[c + 1]; q++) {
            uint32_t e = elements_by_color[q];
            for (int k = 0; k < npe; k++) {
                int b = (int)el[e * npe + k] * 3;
                dofs[k * 3] = b; dofs[k * 3 + 1] = b + 1; dofs[k * 3 + 2] = b + 2;
            }
            for (int j = 0; j < nd; j++) xl[j] = x[dofs[j]];
            const double *Ke = ke_all + (size_t)e * kk;
            for (int row = 0; row < nd; row++) {
                double sum = 0;
                for (int col = 0; col < nd; col++) sum += Ke[row * nd + col] * xl[col];
                yl[row] = R(mode, sum);
            }
            for (int j = 0; j < nd; j++) y[dofs[j]] = R(mode, y[dofs[j]] + yl[j]);
        }
    }
    for (int i = 0; i < Nn * 3; i++)
        if (cons[i]) y[i] = x[i];
}

/* ------------------------------------------------------------------------ */
/* pcg.ts:98-215 solvePCG                                                   */
/* ------------------------------------------------------------------------ */

typedef void (*or_apply_fn)(void *ctx, const double *x, double *y);

static double dotv(int n, const double *a, const double *b) {
    double s = 0;
    for (int i = 0; i < n; i++) s += a[i] * b[i];
    return s;
}

typedef struct {
    int n, Nn;
    const double *scalarM; /* PCGOptions.preconditioner (nullable) */
    const double *blockM;  /* PCGOptions.blockPreconditioner (nullable) */
    int mode;
} or_pcg_pre;

static void pcg_apply_pre(const or_pcg_pre *P, const double *r, double *z) {
    if (P->blockM) {
        or_block_precond(P->Nn, P->blockM, r, z, P->mode);
    } else if (P->scalarM) {
        for (int i = 0; i < P->n; i++)
            z[i] = P->scalarM[i] > 1e-30 ? R(P->mode, r[i] / P->scalarM[i]) : r[i];
    } else {
        for (int i = 0; i < P->n; i++) z[i] = r[i];
    }
}

/* Returns 0.  iters/final_res/converged mirror PCGResult. */
static int pcg_core(int n, or_apply_fn applyK, void *kctx, const or_pcg_pre *P, const double *b,
                    double tol, int maxit, int mode, double *x, int *iters, double *final_res,
                    int *converged) {
    double *r = (double *)calloc((size_t)n, sizeof(double));
    double *z = (double *)calloc((size_t)n, sizeof(double));
    double *p = (double *)calloc((size_t)n, sizeof(double));
    double *Ap = (double *)calloc((size_t)n, sizeof(double));
    for (int i = 0; i < n; i++) { x[i] = 0.0; r[i] = b[i]; }
    double b_norm = sqrt(dotv(n, b, b));
    if (b_norm < 1e-30) {
        *iters = 0; *final_res = 0; *converged = 1;
        goto done;
    }
    pcg_apply_pre(P, r, z);
    for (int i = 0; i < n; i++) p[i] = z[i];
    double rz = dotv(n, r, z);
    for (int it = 0; it < maxit; it++) {
        applyK(kctx, p, Ap);
        double pAp = dotv(n, p, Ap);
        if (fabs(pAp) < 1e-30) {
            *iters = it + 1; *final_res = sqrt(dotv(n, r, r)); *converged = 0;
            goto done;
        }
        double alpha = rz / pAp;
        for (int i = 0; i < n; i++) x[i] = R(mode, x[i] + alpha * p[i]);
        for (int i = 0; i < n; i++) r[i] = R(mode, r[i] + -alpha * Ap[i]);
        double rn = sqrt(dotv(n, r, r));
        if (rn < tol || rn / b_norm < tol) {
            *iters = it + 1; *final_res = rn; *converged = 1;
            goto done;
        }
        pcg_apply_pre(P, r, z);
        double rz_new = dotv(n, r, z);
        double beta = rz_new / rz;
        for (int i = 0; i < n; i++) p[i] = R(mode, z[i] + beta * p[i]);
        rz = rz_new;
    }
    *iters = maxit; *final_res = sqrt(dotv(n, r, r)); *converged = 0;
done:
    free(r); free(z); free(p); free(Ap);
    return 0;
}

typedef struct {
    int Nn, npe, ncolors;
    const uint32_t *el;
    const double *ke_all;
    const int *color_offsets;
    const uint32_t *ebc;
    const uint8_t *cons;
    int mode;
} or_k_ctx;

static void k_apply_cb(void *vctx, const double *x, double *y) {
    or_k_ctx *k = (or_k_ctx *)vctx;
    or_apply_k(k->Nn, k->npe, k->el, k->ke_all, k->ncolors, k->color_offsets, k->ebc, k->cons, x,
               y, k->mode);
}

/* solvePCG(applyGlobalK, b, {blockPreconditioner}) as solvePlate calls it
 * (solver.ts:531-542).  bd_inv: inverted block diagonal (9 per node). */
int or_solve_pcg(int Nn, int npe, const uint32_t *el, const double *ke_all, int ncolors,
                 const int *color_offsets, const uint32_t *ebc, const uint8_t *cons,
                 const double *bd_inv, const double *b, double tol, int maxit, int mode, double *x,
                 int *iters, double *final_res, int *converged) {
    or_k_ctx k = {Nn, npe, ncolors, el, ke_all, color_offsets, ebc, cons, mode};
    or_pcg_pre P = {Nn * 3, Nn, NULL, bd_inv, mode};
    return pcg_core(Nn * 3, k_apply_cb, &k, &P, b, tol, maxit, mode, x, iters, final_res,
                    converged);
}

/* solveTestSystem, pcg.ts:221-247 (known answer x = ones(10)) */
static void tridiag_cb(void *vctx, const double *x, double *y) {
    (void)vctx;
    int n = 10;
    for (int i = 0; i < n; i++) {
        y[i] = (double)(float)(2 * x[i]);
        if (i > 0) y[i] = (double)(float)(y[i] - x[i - 1]);
        if (i < n - 1) y[i] = (double)(float)(y[i] - x[i + 1]);
    }
}

int or_solve_test_system(double *x10, int *iters, double *final_res, int *converged) {
    double b[10] = {0}, M[10];
    b[0] = 1; b[9] = 1;
    for (int i = 0; i < 10; i++) M[i] = 2;
    or_pcg_pre P = {10, 0, M, NULL, OR_REF};
    return pcg_core(10, tridiag_cb, NULL, &P, b, 1e-10, 100, OR_REF, x10, iters, final_res,
                    converged);
}

/* ------------------------------------------------------------------------ */
/* FP64 truth: assembled CSR of the constrained operator                    */
/* ------------------------------------------------------------------------ */

/* Assembles A = K_ff (+) I_cc as COO triplets (duplicates summed by the
 * caller).  Constrained rows and columns are dropped from K and a unit
 * diagonal is put on each constrained DOF; for F with zero constrained
 * entries this has the same solution as the reference operator
 * (solver.ts:479-482).  Returns the number of triplets written; call with
 * rows == NULL to count. */
long or_assemble_coo(int Nn, int Ne, int npe, const uint32_t *el, const double *ke_all,
                     const uint8_t *cons, int *rows, int *cols, double *vals) {
    int nd = 3 * npe, kk = nd * nd;
    long m = 0;
    for (int e = 0; e < Ne; e++) {
        const double *Ke = ke_all + (size_t)e * kk;
        for (int i = 0; i < nd; i++) {
            int gi = (int)el[e * npe + i / 3] * 3 + i % 3;
            if (cons[gi]) continue;
            for (int j = 0; j < nd; j++) {
                int gj = (int)el[e * npe + j / 3] * 3 + j % 3;
                if (cons[gj]) continue;
                if (rows) { rows[m] = gi; cols[m] = gj; vals[m] = Ke[i * nd + j]; }
                m++;
            }
        }
    }
    for (int i = 0; i < Nn * 3; i++) {
        if (!cons[i]) continue;
        if (rows) { rows[m] = i; cols[m] = i; vals[m] = 1.0; }
        m++;
    }
    return m;
}

/* ------------------------------------------------------------------------ */
/* postprocess.ts: nodal bending moments                                    */
/* ------------------------------------------------------------------------ */

/* computeMoments (postprocess.ts:40-54) with computeMomentsQuad (:59-157)
 * and computeMomentsTriangle (:164-264): curvatures at the element centroid
 * (Q4: shape derivatives at xi = eta = 0 through the Jacobian,
 * element.ts:80-184; DKT: linear-triangle derivatives, stored in a
 * Float32Array in the reference), moments with the plate's D and nu, summed
 * into the element's nodes in element order (Float32Array accumulators) and
 * averaged.  x: displacements [3 Nn] (a Float32Array in the reference).
 * Triangles with |2A| < 1e-15 are skipped (:199). */
void or_moments(int Nn, int Ne, int npe, const float *nodes, const uint32_t *el, double E, double nu,
                double t, const double *x, int mode, double *Mx, double *My, double *Mxy) {
    const double D = flexural_rigidity(E, nu, t);
    double *sx = calloc((size_t)Nn, sizeof(double)), *sy = calloc((size_t)Nn, sizeof(double));
    double *sxy = calloc((size_t)Nn, sizeof(double)), *cnt = calloc((size_t)Nn, sizeof(double));
    for (int e = 0; e < Ne; e++) {
        const uint32_t *en = el + (size_t)e * npe;
        double dNdx[4], dNdy[4];
        if (npe == 4) {
            float c[8];
            for (int i = 0; i < 4; i++) {
                c[2 * i] = nodes[2 * en[i]];
                c[2 * i + 1] = nodes[2 * en[i] + 1];
            }
            double dNdXi[4], dNdEta[4];
            shape_derivs(0.0, 0.0, dNdXi, dNdEta);
            phys_derivs(c, dNdXi, dNdEta, dNdx, dNdy);
        } else {
            const double x1 = nodes[2 * en[0]], y1 = nodes[2 * en[0] + 1];
            const double x2 = nodes[2 * en[1]], y2 = nodes[2 * en[1] + 1];
            const double x3 = nodes[2 * en[2]], y3 = nodes[2 * en[2] + 1];
            const double twoA = (x2 - x1) * (y3 - y1) - (x3 - x1) * (y2 - y1);
            if (fabs(twoA) < 1e-15) continue;
            const double inv = 1 / twoA;
            dNdx[0] = R(mode, (y2 - y3) * inv); dNdy[0] = R(mode, (x3 - x2) * inv);
            dNdx[1] = R(mode, (y3 - y1) * inv); dNdy[1] = R(mode, (x1 - x3) * inv);
            dNdx[2] = R(mode, (y1 - y2) * inv); dNdy[2] = R(mode, (x2 - x1) * inv);
        }
        double kx = 0, ky = 0, kxy = 0;
        for (int i = 0; i < npe; i++) {
            const double tx = R(mode, x[3 * (size_t)en[i] + 1]), ty = R(mode, x[3 * (size_t)en[i] + 2]);
            kx += dNdx[i] * ty;
            ky += -dNdy[i] * tx;
            kxy += dNdy[i] * ty - dNdx[i] * tx;
        }
        const double mx = D * (kx + nu * ky), my = D * (ky + nu * kx), mxy = (D * (1 - nu) * kxy) / 2;
        for (int i = 0; i < npe; i++) {
            const uint32_t n = en[i];
            sx[n] = R(mode, sx[n] + mx);
            sy[n] = R(mode, sy[n] + my);
            sxy[n] = R(mode, sxy[n] + mxy);
            cnt[n] = R(mode, cnt[n] + 1);
        }
    }
    for (int n = 0; n < Nn; n++) {
        Mx[n] = cnt[n] > 0 ? R(mode, sx[n] / cnt[n]) : 0.0;
        My[n] = cnt[n] > 0 ? R(mode, sy[n] / cnt[n]) : 0.0;
        Mxy[n] = cnt[n] > 0 ? R(mode, sxy[n] / cnt[n]) : 0.0;
    }
    free(sx); free(sy); free(sxy); free(cnt);
}
