// Element stiffness matrices in FP64 on the device.
//
// Q4 Mindlin (12x12) follows computeElementStiffness, element.ts:258-483:
// 2x2 Gauss bending (points +-1/sqrt(3), weight 1) with
// Db = D [[1, nu, 0], [nu, 1, 0], [0, 0, (1-nu)/2]], D = E t^3 / 12(1-nu^2),
// curvatures kx = dthy/dx, ky = -dthx/dy, kxy = dthy/dy - dthx/dx; and
// 1-point shear at the centre (weight 4) with Ds = kappa G t, kappa = 5/6,
// gxz = dw/dx + thy, gyz = dw/dy - thx.
//
// DKT (9x9) follows computeDKTStiffness, element.ts:642-943 exactly as the
// reference writes it (its B rows and Hx/Hy derivative table included), so
// the GPU applies the same operator as the reference CPU solver.
//
// DOF order per element: [w0, thx0, thy0, w1, ...]; Ke is row-major.
#pragma once

namespace pg {

__host__ __device__ inline double flexural_rigidity(double E, double nu, double t) {
    return (E * t * t * t) / (12.0 * (1.0 - nu * nu));
}

// Physical shape-function derivatives of the Q4 element at (xi, eta);
// returns det J.  (element.ts:80-184)
__device__ __forceinline__ double q4_derivs(const double* __restrict__ c, double xi, double eta,
                                            double* __restrict__ dNdx, double* __restrict__ dNdy) {
    const double xm = 1 - xi, xp = 1 + xi, em = 1 - eta, ep = 1 + eta;
    const double dxi[4] = {-em * 0.25, em * 0.25, ep * 0.25, -ep * 0.25};
    const double deta[4] = {-xm * 0.25, -xp * 0.25, xp * 0.25, xm * 0.25};
    double J11 = 0, J12 = 0, J21 = 0, J22 = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        J11 += dxi[k] * c[2 * k];
        J12 += dxi[k] * c[2 * k + 1];
        J21 += deta[k] * c[2 * k];
        J22 += deta[k] * c[2 * k + 1];
    }
    const double det = J11 * J22 - J12 * J21;
    const double inv = 1.0 / det;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        dNdx[k] = inv * (J22 * dxi[k] - J12 * deta[k]);
        dNdy[k] = inv * (-J21 * dxi[k] + J11 * deta[k]);
    }
    return det;
}

// coords: x0,y0,x1,y1,... (the mesh's float32 values, widened)
__device__ inline void q4_ke(const double* __restrict__ c, double E, double nu, double t,
                             double* __restrict__ Ke) {
    const double gp = 0.5773502691896257;
    const double D = flexural_rigidity(E, nu, t);
    const double D11 = D, D12 = D * nu, D22 = D, D33 = D * (1.0 - nu) * 0.5;
    const double Dsc = (5.0 / 6.0) * (E / (2.0 * (1.0 + nu))) * t;
    for (int i = 0; i < 144; i++) Ke[i] = 0.0;

    const double sx[4] = {-1, 1, 1, -1}, sy[4] = {-1, -1, 1, 1};
    for (int g = 0; g < 4; g++) {
        double dNdx[4], dNdy[4];
        const double f = fabs(q4_derivs(c, sx[g] * gp, sy[g] * gp, dNdx, dNdy));
        for (int i = 0; i < 4; i++) {
            for (int j = 0; j < 4; j++) {
                const int tx_i = 3 * i + 1, ty_i = 3 * i + 2, tx_j = 3 * j + 1, ty_j = 3 * j + 2;
                Ke[tx_i * 12 + tx_j] += f * (dNdy[i] * D22 * dNdy[j] + dNdx[i] * D33 * dNdx[j]);
                Ke[ty_i * 12 + ty_j] += f * (dNdx[i] * D11 * dNdx[j] + dNdy[i] * D33 * dNdy[j]);
                Ke[tx_i * 12 + ty_j] += f * (-dNdy[i] * D12 * dNdx[j] - dNdx[i] * D33 * dNdy[j]);
                Ke[ty_i * 12 + tx_j] += f * (-dNdx[i] * D12 * dNdy[j] - dNdy[i] * D33 * dNdx[j]);
            }
        }
    }
    {
        double dNdx[4], dNdy[4];
        const double f = 4.0 * fabs(q4_derivs(c, 0.0, 0.0, dNdx, dNdy));
        const double N = 0.25;  // every Q4 shape function at the centre
        for (int i = 0; i < 4; i++) {
            for (int j = 0; j < 4; j++) {
                const int w_i = 3 * i, tx_i = 3 * i + 1, ty_i = 3 * i + 2;
                const int w_j = 3 * j, tx_j = 3 * j + 1, ty_j = 3 * j + 2;
                Ke[w_i * 12 + w_j] += f * (dNdx[i] * Dsc * dNdx[j] + dNdy[i] * Dsc * dNdy[j]);
                Ke[w_i * 12 + tx_j] += f * (dNdy[i] * Dsc * (-N));
                Ke[w_i * 12 + ty_j] += f * (dNdx[i] * Dsc * N);
                Ke[tx_i * 12 + w_j] += f * ((-N) * Dsc * dNdy[j]);
                Ke[tx_i * 12 + tx_j] += f * (N * Dsc * N);
                Ke[ty_i * 12 + w_j] += f * (N * Dsc * dNdx[j]);
                Ke[ty_i * 12 + ty_j] += f * (N * Dsc * N);
            }
        }
    }
}

__device__ inline void dkt_ke(const double* __restrict__ c, double E, double nu, double t,
                              double* __restrict__ Ke) {
    for (int i = 0; i < 81; i++) Ke[i] = 0.0;
    const double x1 = c[0], y1 = c[1], x2 = c[2], y2 = c[3], x3 = c[4], y3 = c[5];
    const double x12 = x1 - x2, y12 = y1 - y2, x23 = x2 - x3, y23 = y2 - y3;
    const double x31 = x3 - x1, y31 = y3 - y1;
    const double L12 = x12 * x12 + y12 * y12, L23 = x23 * x23 + y23 * y23;
    const double L31 = x31 * x31 + y31 * y31;
    const double twoA = x12 * y31 - x31 * y12;
    const double area = fabs(twoA) * 0.5;
    if (area < 1e-15) return;  // degenerate triangle: zero stiffness
    const double D = flexural_rigidity(E, nu, t);
    const double D11 = D, D12 = D * nu, D22 = D, D33 = D * (1.0 - nu) * 0.5;

    const double a4 = -x23 / L23, b4 = 3 * x23 * y23 / (4 * L23);
    const double c4 = (x23 * x23 - 2 * y23 * y23) / (4 * L23), d4 = -y23 / L23;
    const double e4 = (y23 * y23 - 2 * x23 * x23) / (4 * L23);
    const double a5 = -x31 / L31, b5 = 3 * x31 * y31 / (4 * L31);
    const double c5 = (x31 * x31 - 2 * y31 * y31) / (4 * L31), d5 = -y31 / L31;
    const double e5 = (y31 * y31 - 2 * x31 * x31) / (4 * L31);
    const double a6 = -x12 / L12, b6 = 3 * x12 * y12 / (4 * L12);
    const double c6 = (x12 * x12 - 2 * y12 * y12) / (4 * L12), d6 = -y12 / L12;
    const double e6 = (y12 * y12 - 2 * x12 * x12) / (4 * L12);
    const double P4 = -6 * a4, P5 = -6 * a5, P6 = -6 * a6;
    const double t4 = -6 * d4, t5 = -6 * d5, t6 = -6 * d6;
    const double q4 = 3 * a4, q5 = 3 * a5, q6 = 3 * a6;
    const double r4 = 3 * d4, r5 = 3 * d5, r6 = 3 * d6;
    const double inv2A = 1.0 / twoA;
    const double L1s[3] = {1.0 / 6, 2.0 / 3, 1.0 / 6}, L2s[3] = {1.0 / 6, 1.0 / 6, 2.0 / 3};

    for (int g = 0; g < 3; g++) {
        const double L1 = L1s[g], L2 = L2s[g];
        const double m1 = 1 - 2 * L1, m2 = 1 - 2 * L2;
        double hx1[9], hx2[9], hy1[9], hy2[9];
        // d(beta_x)/dL1, d(beta_x)/dL2 (element.ts:859-884)
        hx1[0] = P6 * m1 + (P5 - P6) * L2;
        hx1[1] = q6 * m1 - (q5 + q6) * L2;
        hx1[2] = -4 + 6 * (L1 + L2) + (c5 - c6) * L2 + c6 * m1;
        hx2[0] = -P6 * m2 + (P4 - P5) * L1 - P5 * m2;
        hx2[1] = q6 * m2 - (q4 + q5) * L1 + q5 * m2;
        hx2[2] = -4 + 6 * (L1 + L2) + (c4 - c5) * L1 + c5 * m2;
        hx1[3] = P4 * L2 + P6 * m1;
        hx1[4] = q4 * L2 - q6 * m1;
        hx1[5] = c4 * L2 - c6 * m1;
        hx2[3] = P4 * m2 + P5 * L1;
        hx2[4] = q4 * m2 - q5 * L1;
        hx2[5] = c4 * m2 - c5 * L1;
        hx1[6] = -P5 * L2 - P6 * m1;
        hx1[7] = q5 * L2 + q6 * m1;
        hx1[8] = -c5 * L2 + c6 * m1;
        hx2[6] = -P4 * L1 - P5 * m2;
        hx2[7] = q4 * L1 + q5 * m2;
        hx2[8] = -c4 * L1 + c5 * m2;
        // d(beta_y)/dL1, d(beta_y)/dL2 (element.ts:915-940)
        hy1[0] = t6 * m1 + (t5 - t6) * L2;
        hy1[1] = 1 + r6 * m1 - (r5 + r6) * L2;
        hy1[2] = -e6 * m1 + (b5 - b6) * L2;
        hy2[0] = -t6 * m2 + (t4 - t5) * L1 - t5 * m2;
        hy2[1] = 1 + r6 * m2 - (r4 + r5) * L1 + r5 * m2;
        hy2[2] = e6 * m2 + (b4 - b5) * L1 - b5 * m2;
        hy1[3] = t4 * L2 + t6 * m1;
        hy1[4] = -1 + r4 * L2 - r6 * m1;
        hy1[5] = -e4 * L2 - b6 * m1;
        hy2[3] = t4 * m2 + t5 * L1;
        hy2[4] = -1 + r4 * m2 - r5 * L1;
        hy2[5] = -e4 * m2 + b5 * L1;
        hy1[6] = -t5 * L2 - t6 * m1;
        hy1[7] = r5 * L2 + r6 * m1;
        hy1[8] = e5 * L2 + b6 * m1;
        hy2[6] = -t4 * L1 - t5 * m2;
        hy2[7] = r4 * L1 + r5 * m2;
        hy2[8] = e4 * L1 - b5 * m2;

        double B[27], DB[27];
        for (int j = 0; j < 9; j++) {
            B[j] = inv2A * ((-y23) * hx1[j] + (-y31) * hx2[j]);
            B[9 + j] = inv2A * (x23 * hy1[j] + x31 * hy2[j]);
            B[18 + j] = inv2A * (x23 * hx1[j] + x31 * hx2[j] + (-y23) * hy1[j] + (-y31) * hy2[j]);
        }
        for (int j = 0; j < 9; j++) {
            DB[j] = D11 * B[j] + D12 * B[9 + j];
            DB[9 + j] = D12 * B[j] + D22 * B[9 + j];
            DB[18 + j] = D33 * B[18 + j];
        }
        const double f = area / 3.0;
        for (int i = 0; i < 9; i++)
            for (int j = 0; j < 9; j++)
                Ke[i * 9 + j] += f * (B[i] * DB[j] + B[9 + i] * DB[9 + j] + B[18 + i] * DB[18 + j]);
    }
}

}  // namespace pg
