// The unit-modulus hex8 element stiffness of the reference (host code), shared by the library and by
// gen_ke_pattern.cpp, which derives the FP64 streaming kernel's coefficient pattern from its bits.
#pragma once
#include <cmath>
#include <cstring>

namespace t3d {

// Unit-modulus hex8 stiffness (fea.cpp:117-179): 2x2x2 Gauss, Voigt [xx,yy,zz,yz,xz,xy],
// local DOF 3a+c with the natural-coordinate node order (-,-,-),(+,-,-),(+,+,-),(-,+,-), then +z.
inline void hex8_stiffness(double nu, double h, double* Ke) {
    const double lam = nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    const double mu = 1.0 / (2.0 * (1.0 + nu));
    double D[6][6] = {{0}};
    for (int i = 0; i < 3; ++i) {
        for (int j = 0; j < 3; ++j) D[i][j] = lam;
        D[i][i] = lam + 2.0 * mu;
        D[3 + i][3 + i] = mu;
    }
    static const double sg[8] = {-1, 1, 1, -1, -1, 1, 1, -1};
    static const double tg[8] = {-1, -1, 1, 1, -1, -1, 1, 1};
    static const double pg[8] = {-1, -1, -1, -1, 1, 1, 1, 1};
    const double gq = 1.0 / std::sqrt(3.0);
    const double detJ = (h * h * h) / 8.0, sc = 2.0 / h;
    std::memset(Ke, 0, 576 * sizeof(double));
    for (int a = 0; a < 2; ++a)
        for (int b = 0; b < 2; ++b)
            for (int c = 0; c < 2; ++c) {
                const double s = a ? gq : -gq, t = b ? gq : -gq, q = c ? gq : -gq;
                double B[6][24] = {{0}};
                for (int n = 0; n < 8; ++n) {
                    const double dx = 0.125 * sg[n] * (1 + tg[n] * t) * (1 + pg[n] * q) * sc;
                    const double dy = 0.125 * tg[n] * (1 + sg[n] * s) * (1 + pg[n] * q) * sc;
                    const double dz = 0.125 * pg[n] * (1 + sg[n] * s) * (1 + tg[n] * t) * sc;
                    B[0][3 * n] = dx; B[1][3 * n + 1] = dy; B[2][3 * n + 2] = dz;
                    B[3][3 * n + 1] = dz; B[3][3 * n + 2] = dy;
                    B[4][3 * n] = dz; B[4][3 * n + 2] = dx;
                    B[5][3 * n] = dy; B[5][3 * n + 1] = dx;
                }
                double DB[6][24];
                for (int i = 0; i < 6; ++i)
                    for (int j = 0; j < 24; ++j) {
                        double acc = 0.0;
                        for (int k = 0; k < 6; ++k) acc += D[i][k] * B[k][j];
                        DB[i][j] = acc;
                    }
                for (int i = 0; i < 24; ++i)
                    for (int j = 0; j < 24; ++j) {
                        double acc = 0.0;
                        for (int k = 0; k < 6; ++k) acc += B[k][i] * DB[k][j];
                        Ke[i * 24 + j] += acc * detJ;
                    }
            }
}

}  // namespace t3d
