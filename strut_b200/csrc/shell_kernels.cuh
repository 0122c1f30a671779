// ShellMITC4 on an ElasticMembranePlateSection (elements/shell4.mojo:10-363), linear: its
// 24 x 24 global stiffness is computed once per shell at handle creation into the element
// stiffness array (the band gathers read it like a frame element's k), and every Newton
// iteration its internal force f = K u_e is formed after the frame elements' state
// determination (stiffness_internal_surface.mojo:240-280).
#pragma once

#include "kernels.cuh"

namespace strut {

struct DevShell {
    int dof[24];          // absolute u_full indices, nodes in order
    long long ek_off;     // 576 stiffness entries (row-major) in the element stiffness array
    long long ef_off;     // 24 force entries in the element force array
    double x[4], y[4], z[4];
    double E, nu, h;
};

// MITC4 basis g1, g2, g3 from the diagonals, local coordinates, membrane / bending /
// transverse-shear moduli, assumed transverse-shear strains through the edge interpolation,
// 2 x 2 Gauss points, B projected through Gmem / Gshear, drilling with Ktt = G h; the bending
// block of dd negated and the bending rows of B flipped back, as the reference does.  Returns 1
// on a singular Jacobian.
__device__ __forceinline__ void shell_normalize(double* x, double* y, double* z) {
    const double n = sqrt(*x * *x + *y * *y + *z * *z);
    *x /= n;
    *y /= n;
    *z /= n;
}

__device__ int shell4_stiffness(double E, double nu, double h, const double* x, const double* y, const double* z,
                                double* K) {
    double v1x = (x[2] + x[1] - x[3] - x[0]) * 0.5, v1y = (y[2] + y[1] - y[3] - y[0]) * 0.5,
           v1z = (z[2] + z[1] - z[3] - z[0]) * 0.5;
    double v2x = (x[3] + x[2] - x[1] - x[0]) * 0.5, v2y = (y[3] + y[2] - y[1] - y[0]) * 0.5,
           v2z = (z[3] + z[2] - z[1] - z[0]) * 0.5;
    double g1x = v1x, g1y = v1y, g1z = v1z;
    shell_normalize(&g1x, &g1y, &g1z);
    const double alpha = v2x * g1x + v2y * g1y + v2z * g1z;
    v2x -= alpha * g1x;
    v2y -= alpha * g1y;
    v2z -= alpha * g1z;
    double g2x = v2x, g2y = v2y, g2z = v2z;
    shell_normalize(&g2x, &g2y, &g2z);
    const double g3x = g1y * g2z - g1z * g2y, g3y = g1z * g2x - g1x * g2z, g3z = g1x * g2y - g1y * g2x;
    double xl[2][4];
    for (int i = 0; i < 4; ++i) {
        xl[0][i] = x[i] * g1x + y[i] * g1y + z[i] * g1z;
        xl[1][i] = x[i] * g2x + y[i] * g2y + z[i] * g2z;
    }
    const double factor = E / (1.0 - nu * nu);
    const double Dm[3][3] = {{factor, factor * nu, 0.0}, {factor * nu, factor, 0.0}, {0.0, 0.0, factor * (1.0 - nu) / 2.0}};
    const double bf = E * h * h * h / (12.0 * (1.0 - nu * nu));
    const double Db[3][3] = {{bf, bf * nu, 0.0}, {bf * nu, bf, 0.0}, {0.0, 0.0, bf * (1.0 - nu) / 2.0}};
    const double G = E / (2.0 * (1.0 + nu));
    const double Ds = (5.0 / 6.0) * G * h;
    const double Ktt = G * h;
    double dd[8][8] = {{0}};
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            dd[i][j] = Dm[i][j] * h;
            dd[i + 3][j + 3] = -Db[i][j];
        }
    dd[6][6] = Ds;
    dd[7][7] = Ds;
    const double dx34 = xl[0][2] - xl[0][3], dy34 = xl[1][2] - xl[1][3];
    const double dx21 = xl[0][1] - xl[0][0], dy21 = xl[1][1] - xl[1][0];
    const double dx32 = xl[0][2] - xl[0][1], dy32 = xl[1][2] - xl[1][1];
    const double dx41 = xl[0][3] - xl[0][0], dy41 = xl[1][3] - xl[1][0];
    double Gm[4][12] = {{0}};
    const double q4 = 0.25;
    Gm[0][0] = -0.5; Gm[0][1] = -dy41 * q4; Gm[0][2] = dx41 * q4;
    Gm[0][9] = 0.5;  Gm[0][10] = -dy41 * q4; Gm[0][11] = dx41 * q4;
    Gm[1][0] = -0.5; Gm[1][1] = -dy21 * q4; Gm[1][2] = dx21 * q4;
    Gm[1][3] = 0.5;  Gm[1][4] = -dy21 * q4; Gm[1][5] = dx21 * q4;
    Gm[2][3] = -0.5; Gm[2][4] = -dy32 * q4; Gm[2][5] = dx32 * q4;
    Gm[2][6] = 0.5;  Gm[2][7] = -dy32 * q4; Gm[2][8] = dx32 * q4;
    Gm[3][6] = 0.5;  Gm[3][7] = -dy34 * q4; Gm[3][8] = dx34 * q4;
    Gm[3][9] = -0.5; Gm[3][10] = -dy34 * q4; Gm[3][11] = dx34 * q4;
    const double Ax = -xl[0][0] + xl[0][1] + xl[0][2] - xl[0][3];
    const double Bx = xl[0][0] - xl[0][1] + xl[0][2] - xl[0][3];
    const double Cx = -xl[0][0] - xl[0][1] + xl[0][2] + xl[0][3];
    const double Ay = -xl[1][0] + xl[1][1] + xl[1][2] - xl[1][3];
    const double By = xl[1][0] - xl[1][1] + xl[1][2] - xl[1][3];
    const double Cy = -xl[1][0] - xl[1][1] + xl[1][2] + xl[1][3];
    const double alph = atan2(Ay, Ax);
    const double beta = 0.5 * 3.141592653589793 - atan2(Cx, Cy);
    const double Rot[2][2] = {{sin(beta), -sin(alph)}, {-cos(beta), cos(alph)}};
    const double r3i = 1.0 / sqrt(3.0);
    const double sg[4] = {-r3i, r3i, r3i, -r3i}, tg[4] = {-r3i, -r3i, r3i, r3i};
    const double sn[4] = {-0.5, 0.5, 0.5, -0.5}, tn[4] = {-0.5, -0.5, 0.5, 0.5};
    const double Gmem[2][3] = {{g1x, g1y, g1z}, {g2x, g2y, g2z}};
    const double Gshear[3][6] = {{g3x, g3y, g3z, 0, 0, 0}, {0, 0, 0, g1x, g1y, g1z}, {0, 0, 0, g2x, g2y, g2z}};
    for (int t = 0; t < 576; ++t) K[t] = 0.0;
    for (int gp = 0; gp < 4; ++gp) {
        const double ss = sg[gp], tt = tg[gp];
        double shp[3][4];
        for (int i = 0; i < 4; ++i) {
            shp[2][i] = (0.5 + sn[i] * ss) * (0.5 + tn[i] * tt);
            shp[0][i] = sn[i] * (0.5 + tn[i] * tt);
            shp[1][i] = tn[i] * (0.5 + sn[i] * ss);
        }
        double xs[2][2];
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 2; ++j) {
                xs[i][j] = 0.0;
                for (int k = 0; k < 4; ++k) xs[i][j] += xl[i][k] * shp[j][k];
            }
        const double xsj = xs[0][0] * xs[1][1] - xs[0][1] * xs[1][0];
        if (xsj == 0.0) return 1;
        const double jinv = 1.0 / xsj;
        const double sx00 = xs[1][1] * jinv, sx11 = xs[0][0] * jinv, sx01 = -xs[0][1] * jinv,
                     sx10 = -xs[1][0] * jinv;
        for (int i = 0; i < 4; ++i) {
            const double temp = shp[0][i] * sx00 + shp[1][i] * sx10;
            shp[1][i] = shp[0][i] * sx01 + shp[1][i] * sx11;
            shp[0][i] = temp;
        }
        const double dvol = 1.0 * xsj;
        double Ms[2][4] = {{0}};
        Ms[1][0] = 1.0 - ss;
        Ms[0][1] = 1.0 - tt;
        Ms[1][2] = 1.0 + ss;
        Ms[0][3] = 1.0 + tt;
        double Bsv[2][12];
        for (int i = 0; i < 2; ++i)
            for (int j = 0; j < 12; ++j) {
                double sum = 0.0;
                for (int k = 0; k < 4; ++k) sum += Ms[i][k] * Gm[k][j];
                Bsv[i][j] = sum;
            }
        double r1 = Cx + ss * Bx, r3 = Cy + ss * By;
        r1 = sqrt(r1 * r1 + r3 * r3);
        double r2 = Ax + tt * Bx;
        r3 = Ay + tt * By;
        r2 = sqrt(r2 * r2 + r3 * r3);
        for (int j = 0; j < 12; ++j) {
            Bsv[0][j] = Bsv[0][j] * r1 / (8.0 * xsj);
            Bsv[1][j] = Bsv[1][j] * r2 / (8.0 * xsj);
        }
        double Bs[2][12];
        for (int j = 0; j < 12; ++j) {
            Bs[0][j] = Rot[0][0] * Bsv[0][j] + Rot[0][1] * Bsv[1][j];
            Bs[1][j] = Rot[1][0] * Bsv[0][j] + Rot[1][1] * Bsv[1][j];
        }
        double saveB[4][8][6];
        double Bdrill[4][6];
        for (int j = 0; j < 4; ++j) {
            double Bmem[3][2] = {{0}}, Bb[3][2] = {{0}};
            Bmem[0][0] = shp[0][j];
            Bmem[1][1] = shp[1][j];
            Bmem[2][0] = shp[1][j];
            Bmem[2][1] = shp[0][j];
            Bb[0][1] = -shp[0][j];
            Bb[1][0] = shp[1][j];
            Bb[2][0] = shp[0][j];
            Bb[2][1] = -shp[1][j];
            double Bsh[2][3];
            for (int p = 0; p < 3; ++p) {
                Bsh[0][p] = Bs[0][j * 3 + p];
                Bsh[1][p] = Bs[1][j * 3 + p];
            }
            for (int p = 0; p < 8; ++p)
                for (int q = 0; q < 6; ++q) saveB[j][p][q] = 0.0;
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) {
                    double sm = 0.0, sb = 0.0;
                    for (int r = 0; r < 2; ++r) {
                        sm += Bmem[p][r] * Gmem[r][q];
                        sb += Bb[p][r] * Gmem[r][q];
                    }
                    saveB[j][p][q] = sm;
                    saveB[j][p + 3][q + 3] = sb;
                }
            for (int p = 0; p < 2; ++p)
                for (int q = 0; q < 6; ++q) {
                    double s_ = 0.0;
                    for (int r = 0; r < 3; ++r) s_ += Bsh[p][r] * Gshear[r][q];
                    saveB[j][p + 6][q] = s_;
                }
            const double B1 = -0.5 * shp[1][j], B2 = 0.5 * shp[0][j], B6 = -shp[2][j];
            Bdrill[j][0] = B1 * g1x + B2 * g2x;
            Bdrill[j][1] = B1 * g1y + B2 * g2y;
            Bdrill[j][2] = B1 * g1z + B2 * g2z;
            Bdrill[j][3] = B6 * g3x;
            Bdrill[j][4] = B6 * g3y;
            Bdrill[j][5] = B6 * g3z;
        }
        for (int j = 0; j < 4; ++j) {
            double BJ[8][6];
            for (int p = 0; p < 8; ++p)
                for (int q = 0; q < 6; ++q) BJ[p][q] = saveB[j][p][q];
            for (int p = 3; p < 6; ++p)
                for (int q = 3; q < 6; ++q) BJ[p][q] *= -1.0;
            double BJtD[6][8];
            for (int p = 0; p < 6; ++p)
                for (int q = 0; q < 8; ++q) {
                    double sum = 0.0;
                    for (int r = 0; r < 8; ++r) sum += BJ[r][p] * dd[r][q];
                    BJtD[p][q] = sum * dvol;
                }
            double BdJ[6];
            for (int p = 0; p < 6; ++p) BdJ[p] = Bdrill[j][p] * (Ktt * dvol);
            for (int k = 0; k < 4; ++k)
                for (int p = 0; p < 6; ++p)
                    for (int q = 0; q < 6; ++q) {
                        double sum = 0.0;
                        for (int r = 0; r < 8; ++r) sum += BJtD[p][r] * saveB[k][r][q];
                        K[(j * 6 + p) * 24 + k * 6 + q] += sum + BdJ[p] * Bdrill[k][q];
                    }
        }
    }
    return 0;
}

// One thread per shell (setup, once per handle).
__global__ void shell_stiffness_kernel(const DevShell* __restrict__ shells, int n_shells, double* __restrict__ ek,
                                       int* __restrict__ err) {
    const int s = blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= n_shells) return;
    const DevShell& S = shells[s];
    if (shell4_stiffness(S.E, S.nu, S.h, S.x, S.y, S.z, ek + S.ek_off) != 0) atomicExch(err, 1);
}

// One warp per shell, lane a < 24: f_a = sum_b K_ab u_b (row order).
__global__ void shell_force_kernel(const DevShell* __restrict__ shells, int n_shells, const double* __restrict__ ek,
                                   double* __restrict__ ef, const double* __restrict__ u_full) {
    const int s = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (s >= n_shells) return;
    const DevShell& S = shells[s];
    const double u = lane < 24 ? u_full[S.dof[lane]] : 0.0;
    double f = 0.0;
    for (int b = 0; b < 24; ++b) {
        const double ub = __shfl_sync(0xffffffffu, u, b);
        if (lane < 24) f = fma(ek[S.ek_off + lane * 24 + b], ub, f);
    }
    if (lane < 24) ef[S.ef_off + lane] = f;
}

}  // namespace strut
