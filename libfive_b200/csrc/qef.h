// Quadratic error function (QEF) arithmetic of the dual-contouring mesher
// (octree cells) and contourer (quadtree cells, the *2 functions at the end),
// in FP64, shared by the device kernels and the host.
//
//  * qef_push:     Intersection::push (libfive/include/libfive/render/brep/
//                  dc/intersection.hpp:32-59): normalise the gradient, skip
//                  invalid normals, accumulate A^T A, A^T b, b^T b and the
//                  mass point.
//  * qef_rank:     Intersection::get_rank (intersection.hpp:67-88): number of
//                  eigenvalues of A^T A below EIGENVALUE_CUTOFF (0.1).
//  * qef_vertex:   DCTree::findVertex (libfive/src/render/brep/dc/
//                  dc_tree.inl:740-813): rank-truncated pseudo-inverse
//                  minimisation towards the mass point.
//
// The reference decomposes A^T A with Eigen's SelfAdjointEigenSolver, which
// is not available here; sym3_eigen is a cyclic Jacobi eigensolver (Golub &
// Van Loan, "Matrix Computations", section 8.5) with a fixed sweep order and
// stopping rule, so every caller that compiles this header without FMA
// contraction gets bit-identical eigenpairs on the host and the device.
#pragma once
#include <cmath>

#ifdef __CUDACC__
#define QEF_HD __host__ __device__ __forceinline__
#else
#define QEF_HD inline
using std::isfinite;
using std::sqrt;
using std::fabs;
#endif

namespace lfb {

// Symmetric 3x3 matrices are stored as {xx, xy, xz, yy, yz, zz}.
struct Qef {
    double ata[6];
    double atb[3];
    double btb;
    double mass[4];   // sum of positions, count
};

constexpr double kEigenvalueCutoff = 0.1;   // dc_flags.hpp:12

QEF_HD void qef_zero(Qef& q)
{
    for (int i = 0; i < 6; ++i) q.ata[i] = 0.0;
    for (int i = 0; i < 3; ++i) q.atb[i] = 0.0;
    q.btb = 0.0;
    for (int i = 0; i < 4; ++i) q.mass[i] = 0.0;
}

QEF_HD void qef_add(Qef& q, const Qef& o)
{
    for (int i = 0; i < 6; ++i) q.ata[i] += o.ata[i];
    for (int i = 0; i < 3; ++i) q.atb[i] += o.atb[i];
    q.btb += o.btb;
}

QEF_HD double dot3d(const double* a, const double* b)
{
    return (a[0] * b[0] + a[1] * b[1]) + a[2] * b[2];
}

/// Adds one sample (position, gradient, value) to an edge's QEF.
QEF_HD void qef_push(Qef& q, const double pos[3], const double deriv_in[3],
                     double value)
{
    q.mass[0] += pos[0];
    q.mass[1] += pos[1];
    q.mass[2] += pos[2];
    q.mass[3] += 1.0;
    const double norm = sqrt(dot3d(deriv_in, deriv_in));
    double d[3] = {deriv_in[0] / norm, deriv_in[1] / norm, deriv_in[2] / norm};
    value = value / norm;
    if (norm <= 1e-12 || !isfinite(d[0]) || !isfinite(d[1]) || !isfinite(d[2])) {
        return;
    }
    q.ata[0] += d[0] * d[0];
    q.ata[1] += d[0] * d[1];
    q.ata[2] += d[0] * d[2];
    q.ata[3] += d[1] * d[1];
    q.ata[4] += d[1] * d[2];
    q.ata[5] += d[2] * d[2];
    const double b = dot3d(d, pos) - value;
    q.atb[0] += d[0] * b;
    q.atb[1] += d[1] * b;
    q.atb[2] += d[2] * b;
    q.btb += b * b;
}

/// Eigen-decomposition of a symmetric 3x3 matrix by cyclic Jacobi rotations.
/// evec[r][c]: column c is the eigenvector of eval[c].
QEF_HD void sym3_eigen(const double s[6], double eval[3], double evec[3][3])
{
    double a[3][3] = {{s[0], s[1], s[2]}, {s[1], s[3], s[4]}, {s[2], s[4], s[5]}};
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) evec[r][c] = (r == c) ? 1.0 : 0.0;
    }
    for (int sweep = 0; sweep < 24; ++sweep) {
        const double off = (a[0][1] * a[0][1] + a[0][2] * a[0][2]) + a[1][2] * a[1][2];
        const double diag = (a[0][0] * a[0][0] + a[1][1] * a[1][1]) + a[2][2] * a[2][2];
        if (off == 0.0 || off <= 1e-36 * diag) {
            break;
        }
        for (int pq = 0; pq < 3; ++pq) {
            const int p = (pq == 2) ? 1 : 0;
            const int q = (pq == 0) ? 1 : 2;
            const double apq = a[p][q];
            if (apq == 0.0) {
                continue;
            }
            const double theta = (a[q][q] - a[p][p]) / (2.0 * apq);
            const double t = (theta >= 0.0 ? 1.0 : -1.0) /
                             (fabs(theta) + sqrt(theta * theta + 1.0));
            const double c = 1.0 / sqrt(t * t + 1.0);
            const double sn = t * c;
            const double tau = sn / (1.0 + c);
            a[p][p] -= t * apq;
            a[q][q] += t * apq;
            a[p][q] = 0.0;
            a[q][p] = 0.0;
            const int r = 3 - p - q;
            const double arp = a[r][p], arq = a[r][q];
            a[r][p] = arp - sn * (arq + tau * arp);
            a[p][r] = a[r][p];
            a[r][q] = arq + sn * (arp - tau * arq);
            a[q][r] = a[r][q];
            for (int k = 0; k < 3; ++k) {
                const double vkp = evec[k][p], vkq = evec[k][q];
                evec[k][p] = vkp - sn * (vkq + tau * vkp);
                evec[k][q] = vkq + sn * (vkp - tau * vkq);
            }
        }
    }
    eval[0] = a[0][0];
    eval[1] = a[1][1];
    eval[2] = a[2][2];
}

/// Intersection::get_rank: count of near-zero eigenvalues of A^T A.
QEF_HD int qef_rank(const Qef& q)
{
    double ev[3], U[3][3];
    sym3_eigen(q.ata, ev, U);
    int rank = 0;
    for (int j = 0; j < 3; ++j) rank += (fabs(ev[j]) < kEigenvalueCutoff) ? 1 : 0;
    return rank;
}

/// DCTree::findVertex: writes the vertex, returns the QEF error and, in
/// *rank_out, the number of eigenvalues kept (the feature rank).
QEF_HD double qef_vertex(const Qef& q, double v[3], int* rank_out)
{
    double ev[3], U[3][3];
    sym3_eigen(q.ata, ev, U);
    double D[3];
    int rank = 0;
    for (int i = 0; i < 3; ++i) {
        D[i] = (fabs(ev[i]) < kEigenvalueCutoff) ? 0.0 : (1.0 / ev[i]);
        rank += (D[i] != 0.0) ? 1 : 0;
    }
    if (rank_out) *rank_out = rank;

    // Pseudo-inverse U D U^T
    double P[3][3];
    for (int r = 0; r < 3; ++r) {
        for (int c = 0; c < 3; ++c) {
            P[r][c] = (U[r][0] * D[0] * U[c][0] + U[r][1] * D[1] * U[c][1]) +
                      U[r][2] * D[2] * U[c][2];
        }
    }
    const double A[3][3] = {{q.ata[0], q.ata[1], q.ata[2]},
                            {q.ata[1], q.ata[3], q.ata[4]},
                            {q.ata[2], q.ata[4], q.ata[5]}};
    const double center[3] = {q.mass[0] / q.mass[3], q.mass[1] / q.mass[3],
                              q.mass[2] / q.mass[3]};
    double rhs[3];
    for (int r = 0; r < 3; ++r) {
        rhs[r] = q.atb[r] - dot3d(A[r], center);
    }
    for (int r = 0; r < 3; ++r) {
        v[r] = dot3d(P[r], rhs) + center[r];
    }
    double Av[3];
    for (int r = 0; r < 3; ++r) Av[r] = dot3d(A[r], v);
    return (dot3d(v, Av) - 2.0 * dot3d(v, q.atb)) + q.btb;
}

////////////////////////////////////////////////////////////////////////////////
// The same three operations for quadtree cells (DCTree<2>, Intersection<2>):
// positions and normals in the slice plane, A^T A a symmetric 2x2 matrix
// stored as {xx, xy, yy}.

struct Qef2 {
    double ata[3];
    double atb[2];
    double btb;
    double mass[3];   // sum of positions, count
};

QEF_HD void qef2_zero(Qef2& q)
{
    for (int i = 0; i < 3; ++i) q.ata[i] = 0.0;
    for (int i = 0; i < 2; ++i) q.atb[i] = 0.0;
    q.btb = 0.0;
    for (int i = 0; i < 3; ++i) q.mass[i] = 0.0;
}

QEF_HD void qef2_add(Qef2& q, const Qef2& o)
{
    for (int i = 0; i < 3; ++i) q.ata[i] += o.ata[i];
    for (int i = 0; i < 2; ++i) q.atb[i] += o.atb[i];
    q.btb += o.btb;
}

/// Intersection<2>::push (intersection.hpp:32-59).
QEF_HD void qef2_push(Qef2& q, const double pos[2], const double deriv_in[2], double value)
{
    q.mass[0] += pos[0];
    q.mass[1] += pos[1];
    q.mass[2] += 1.0;
    const double norm = sqrt(deriv_in[0] * deriv_in[0] + deriv_in[1] * deriv_in[1]);
    const double d[2] = {deriv_in[0] / norm, deriv_in[1] / norm};
    value = value / norm;
    if (norm <= 1e-12 || !isfinite(d[0]) || !isfinite(d[1])) {
        return;
    }
    q.ata[0] += d[0] * d[0];
    q.ata[1] += d[0] * d[1];
    q.ata[2] += d[1] * d[1];
    const double b = (d[0] * pos[0] + d[1] * pos[1]) - value;
    q.atb[0] += d[0] * b;
    q.atb[1] += d[1] * b;
    q.btb += b * b;
}

/// Eigen-decomposition of a symmetric 2x2 matrix: one Jacobi rotation (the
/// rotation of sym3_eigen for the pair (0, 1)), which zeroes the
/// off-diagonal term.  evec[r][c]: column c is the eigenvector of eval[c].
QEF_HD void sym2_eigen(const double s[3], double eval[2], double evec[2][2])
{
    double a00 = s[0], a11 = s[2];
    evec[0][0] = 1.0; evec[0][1] = 0.0;
    evec[1][0] = 0.0; evec[1][1] = 1.0;
    const double apq = s[1];
    if (apq != 0.0) {
        const double theta = (a11 - a00) / (2.0 * apq);
        const double t = (theta >= 0.0 ? 1.0 : -1.0) /
                         (fabs(theta) + sqrt(theta * theta + 1.0));
        const double c = 1.0 / sqrt(t * t + 1.0);
        const double sn = t * c;
        const double tau = sn / (1.0 + c);
        a00 -= t * apq;
        a11 += t * apq;
        for (int k = 0; k < 2; ++k) {
            const double vkp = evec[k][0], vkq = evec[k][1];
            evec[k][0] = vkp - sn * (vkq + tau * vkp);
            evec[k][1] = vkq + sn * (vkp - tau * vkq);
        }
    }
    eval[0] = a00;
    eval[1] = a11;
}

/// Intersection<2>::get_rank: count of near-zero eigenvalues of A^T A.
QEF_HD int qef2_rank(const Qef2& q)
{
    double ev[2], U[2][2];
    sym2_eigen(q.ata, ev, U);
    int rank = 0;
    for (int j = 0; j < 2; ++j) rank += (fabs(ev[j]) < kEigenvalueCutoff) ? 1 : 0;
    return rank;
}

/// DCTree<2>::findVertex: writes the vertex, returns the QEF error and, in
/// *rank_out, the number of eigenvalues kept.
QEF_HD double qef2_vertex(const Qef2& q, double v[2], int* rank_out)
{
    double ev[2], U[2][2];
    sym2_eigen(q.ata, ev, U);
    double D[2];
    int rank = 0;
    for (int i = 0; i < 2; ++i) {
        D[i] = (fabs(ev[i]) < kEigenvalueCutoff) ? 0.0 : (1.0 / ev[i]);
        rank += (D[i] != 0.0) ? 1 : 0;
    }
    if (rank_out) *rank_out = rank;
    double P[2][2];
    for (int r = 0; r < 2; ++r) {
        for (int c = 0; c < 2; ++c) {
            P[r][c] = U[r][0] * D[0] * U[c][0] + U[r][1] * D[1] * U[c][1];
        }
    }
    const double A[2][2] = {{q.ata[0], q.ata[1]}, {q.ata[1], q.ata[2]}};
    const double center[2] = {q.mass[0] / q.mass[2], q.mass[1] / q.mass[2]};
    double rhs[2];
    for (int r = 0; r < 2; ++r) {
        rhs[r] = q.atb[r] - (A[r][0] * center[0] + A[r][1] * center[1]);
    }
    for (int r = 0; r < 2; ++r) {
        v[r] = (P[r][0] * rhs[0] + P[r][1] * rhs[1]) + center[r];
    }
    double Av[2];
    for (int r = 0; r < 2; ++r) Av[r] = A[r][0] * v[0] + A[r][1] * v[1];
    return ((v[0] * Av[0] + v[1] * Av[1]) - 2.0 * (v[0] * q.atb[0] + v[1] * q.atb[1])) + q.btb;
}

}  // namespace lfb
