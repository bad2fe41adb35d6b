// Host-side coefficients of the far-field expansion of the demag tensor D = -N.
//
// d^p_x d^q_y d^r_z (1/R) = P_pqr(x, y, z) / R^(2n+1), n = p+q+r, with the integer polynomials
// built by P_{.. +1 ..} = R^2 dP/dx_axis - (2n+1) x_axis P. The averaged tensor over two cells
// of size (hx, hy, hz) is (V/4pi) prod_k (1 + h_k^2 d_k^2/12 + h_k^4 d_k^4/360 + h_k^6 d_k^6/20160)
// applied to d_i d_j (1/R), truncated at total order 8. For each component the result is
// sum over n in {2,4,6,8} of Q_n(u,v,w) / R^(n+1) with (u,v,w) the unit vector; Q_n's
// coefficients are written in the order i = n..0, j = n-i..0 (k = n-i-j) for u^i v^j w^k.
#include "kernels.h"
#include <vector>
#include <cstring>
#include <cmath>

namespace {
const int PD = 9;
struct Poly { double c[PD][PD][PD]; };

void step(const Poly &P, int n, int axis, Poly &out)
{
    memset(&out, 0, sizeof(out));
    for (int i = 0; i < PD; i++)
        for (int j = 0; j < PD; j++)
            for (int k = 0; k < PD; k++) {
                double c = P.c[i][j][k];
                if (c == 0.0) continue;
                int e[3] = {i, j, k};
                if (e[axis] > 0) {
                    int d[3] = {i, j, k};
                    d[axis] -= 1;
                    double dc = c * e[axis];
                    for (int s = 0; s < 3; s++) {
                        int f[3] = {d[0], d[1], d[2]};
                        f[s] += 2;
                        if (f[0] < PD && f[1] < PD && f[2] < PD) out.c[f[0]][f[1]][f[2]] += dc;
                    }
                }
                int g[3] = {i, j, k};
                g[axis] += 1;
                if (g[0] < PD && g[1] < PD && g[2] < PD) out.c[g[0]][g[1]][g[2]] -= (2.0 * n + 1.0) * c;
            }
}
}

void bm_far_coeffs(double hx, double hy, double hz, double *out)
{
    std::vector<Poly> T((size_t)PD * PD * PD);
    auto id = [](int p, int q, int r) { return (size_t)((p * PD + q) * PD + r); };
    memset(&T[id(0, 0, 0)], 0, sizeof(Poly));
    T[id(0, 0, 0)].c[0][0][0] = 1.0;
    for (int p = 0; p < PD; p++)
        for (int q = 0; q < PD; q++)
            for (int r = 0; r < PD; r++) {
                int n = p + q + r;
                if (n > 8 || n == 0) continue;
                if (r > 0) step(T[id(p, q, r - 1)], n - 1, 2, T[id(p, q, r)]);
                else if (q > 0) step(T[id(p, q - 1, 0)], n - 1, 1, T[id(p, q, 0)]);
                else step(T[id(p - 1, 0, 0)], n - 1, 0, T[id(p, 0, 0)]);
            }
    const double C[4] = {1.0, 1.0 / 12.0, 1.0 / 360.0, 1.0 / 20160.0};
    const int comp[6][2] = {{0, 0}, {1, 1}, {2, 2}, {0, 1}, {0, 2}, {1, 2}};
    for (int c = 0; c < 6; c++) {
        double *q = out + c * BM_FARQ_PER_COMP;
        int off = 0;
        for (int o = 0; o < 4; o++) {
            int n = 2 + 2 * o;
            Poly Q;
            memset(&Q, 0, sizeof(Q));
            for (int a = 0; a <= o; a++)
                for (int b = 0; a + b <= o; b++) {
                    int cc = o - a - b;
                    int e[3] = {2 * a, 2 * b, 2 * cc};
                    e[comp[c][0]] += 1;
                    e[comp[c][1]] += 1;
                    double coef = C[a] * C[b] * C[cc] * std::pow(hx, 2 * a) * std::pow(hy, 2 * b) * std::pow(hz, 2 * cc);
                    const Poly &P = T[id(e[0], e[1], e[2])];
                    for (int i = 0; i < PD; i++)
                        for (int j = 0; j < PD; j++)
                            for (int k = 0; k < PD; k++) Q.c[i][j][k] += coef * P.c[i][j][k];
                }
            for (int i = n; i >= 0; i--)
                for (int j = n - i; j >= 0; j--) {
                    int k = n - i - j;
                    q[off++] = Q.c[i][j][k];
                }
        }
    }
}
