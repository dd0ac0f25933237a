/*
 * fm_oracle.c — CPU oracle for the FlexMesh hot path (TEST INFRASTRUCTURE).
 *
 * This file is the checker, never the product: only tests, the smoke check
 * and the benchmark's CPU-baseline leg load it.  It restates, in plain C and
 * single-threaded, the reference's algorithm for the path
 *   unit-cube mesh -> CSR pattern -> element force/tangent -> scatter ->
 *   Dirichlet elimination -> ILU(0) -> PCG -> Newton
 * plus the exact Jacobian and the adjoint, which have no reference code.
 *
 * Floating-point operations follow the reference's order term by term (the
 * file is compiled with -ffp-contract=off), so on x86-64 every FP64 result is
 * bitwise identical to the reference compiled from its own headers; the
 * oracle/_ref build of the reference and the golden fixtures pin that.
 * References are to files of the reference project (FEM/..., CORE/...).
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define ORC_SQRT2 1.41421356237 /* truncated constant, FEM/adaptive_fem_engine.hpp:122,602 */

/* ------------------------------------------------------------------ */
/* A1: structured unit cube, 6 tets per hex                            */
/* FEM/adaptive_fem_engine.hpp:2219-2294                               */
/* ------------------------------------------------------------------ */
/* hex corner offsets and the 6-tet split; these tables fix node and
 * element numbering, so they must equal the reference's (:2240-2247). */
static const int ORC_HEX_CORNER[8][3] = {
    {0, 0, 0}, {1, 0, 0}, {1, 1, 0}, {0, 1, 0},
    {0, 0, 1}, {1, 0, 1}, {1, 1, 1}, {0, 1, 1}};
static const int ORC_TET_OF_HEX[6][4] = {
    {0, 1, 3, 4}, {1, 2, 3, 6}, {1, 3, 4, 6},
    {3, 4, 6, 7}, {1, 4, 5, 6}, {0, 3, 4, 7}};

void orc_unit_cube_sizes(int N, uint32_t* n_nodes, uint32_t* n_elems) {
    uint32_t s = (uint32_t)(N + 1);
    *n_nodes = s * s * s;
    *n_elems = 6u * (uint32_t)N * (uint32_t)N * (uint32_t)N;
}

void orc_unit_cube(int N, double* xyz, uint32_t* conn) {
    const int s = N + 1;
    const double h = 1.0 / N;
    size_t id = 0;
    for (int k = 0; k <= N; ++k)
        for (int j = 0; j <= N; ++j)
            for (int i = 0; i <= N; ++i, ++id) {
                xyz[3 * id + 0] = i * h;
                xyz[3 * id + 1] = j * h;
                xyz[3 * id + 2] = k * h;
            }
    size_t e = 0;
    for (int k = 0; k < N; ++k)
        for (int j = 0; j < N; ++j)
            for (int i = 0; i < N; ++i) {
                uint32_t corner[8];
                for (int c = 0; c < 8; ++c) {
                    int ii = i + ORC_HEX_CORNER[c][0], jj = j + ORC_HEX_CORNER[c][1],
                        kk = k + ORC_HEX_CORNER[c][2];
                    corner[c] = (uint32_t)(kk * s * s + jj * s + ii);
                }
                for (int t = 0; t < 6; ++t, ++e)
                    for (int v = 0; v < 4; ++v) conn[4 * e + v] = corner[ORC_TET_OF_HEX[t][v]];
            }
}

/* |6V| / 6 by the triple product, FEM/mesh_adaptation.hpp:111-126 */
double orc_tet_volume(const double* a, const double* b, const double* c, const double* d) {
    double u[3], v[3], w[3];
    for (int q = 0; q < 3; ++q) { u[q] = b[q] - a[q]; v[q] = c[q] - a[q]; w[q] = d[q] - a[q]; }
    double s6 = u[0] * (v[1] * w[2] - v[2] * w[1]) - u[1] * (v[0] * w[2] - v[2] * w[0]) +
                u[2] * (v[0] * w[1] - v[1] * w[0]);
    return fabs(s6) / 6.0;
}

void orc_volumes(uint32_t n_elems, const double* xyz, const uint32_t* conn, double* vol) {
    for (uint32_t e = 0; e < n_elems; ++e) {
        const uint32_t* c = conn + 4 * (size_t)e;
        vol[e] = orc_tet_volume(xyz + 3 * (size_t)c[0], xyz + 3 * (size_t)c[1],
                                xyz + 3 * (size_t)c[2], xyz + 3 * (size_t)c[3]);
    }
}

/* node -> incident elements, ascending element id (:2279-2291) */
void orc_node_to_elem(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn, uint32_t* ptr,
                      uint32_t* data) {
    memset(ptr, 0, sizeof(uint32_t) * (n_nodes + 1));
    for (size_t q = 0; q < 4 * (size_t)n_elems; ++q) ptr[conn[q] + 1]++;
    for (uint32_t n = 0; n < n_nodes; ++n) ptr[n + 1] += ptr[n];
    uint32_t* fill = (uint32_t*)calloc(n_nodes, sizeof(uint32_t));
    for (uint32_t e = 0; e < n_elems; ++e)
        for (int v = 0; v < 4; ++v) {
            uint32_t n = conn[4 * (size_t)e + v];
            data[ptr[n] + fill[n]++] = e;
        }
    free(fill);
}

/* ------------------------------------------------------------------ */
/* A2/A3: CSR patterns                                                 */
/* FEM/adaptive_fem_engine.hpp:1069-1120                               */
/* ------------------------------------------------------------------ */
/* Sorted unique node neighbour sets (std::set semantics, self included).
 * Returns nbr_ptr[n_nodes+1] and nbr[] (caller frees). */
static void orc_node_neighbours(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn,
                                uint32_t** out_ptr, uint32_t** out_nbr) {
    /* bucket all (node, other) pairs, then sort+unique per node */
    uint32_t* cnt = (uint32_t*)calloc(n_nodes + 1, sizeof(uint32_t));
    for (size_t q = 0; q < 4 * (size_t)n_elems; ++q) cnt[conn[q] + 1] += 4;
    for (uint32_t n = 0; n < n_nodes; ++n) cnt[n + 1] += cnt[n];
    uint32_t* raw = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cnt[n_nodes] + 4);
    uint32_t* fill = (uint32_t*)calloc(n_nodes, sizeof(uint32_t));
    for (uint32_t e = 0; e < n_elems; ++e) {
        const uint32_t* c = conn + 4 * (size_t)e;
        for (int a = 0; a < 4; ++a)
            for (int b = 0; b < 4; ++b) raw[cnt[c[a]] + fill[c[a]]++] = c[b];
    }
    uint32_t* ptr = (uint32_t*)calloc(n_nodes + 1, sizeof(uint32_t));
    uint32_t* nbr = (uint32_t*)malloc(sizeof(uint32_t) * (size_t)cnt[n_nodes] + 4);
    uint32_t w = 0;
    for (uint32_t n = 0; n < n_nodes; ++n) {
        uint32_t b = cnt[n], e = cnt[n + 1];
        /* insertion sort: per-node lists are short (<= 4 * incident elements) */
        for (uint32_t x = b + 1; x < e; ++x) {
            uint32_t v = raw[x];
            uint32_t y = x;
            while (y > b && raw[y - 1] > v) { raw[y] = raw[y - 1]; --y; }
            raw[y] = v;
        }
        ptr[n] = w;
        for (uint32_t x = b; x < e; ++x)
            if (x == b || raw[x] != raw[x - 1]) nbr[w++] = raw[x];
    }
    ptr[n_nodes] = w;
    free(cnt); free(raw); free(fill);
    *out_ptr = ptr;
    *out_nbr = nbr;
}

/* nnz is 9 * sum_n |nb(n)| for both patterns (:1092-1102) */
uint64_t orc_pattern_nnz(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn) {
    uint32_t *ptr, *nbr;
    orc_node_neighbours(n_nodes, n_elems, conn, &ptr, &nbr);
    uint64_t nnz = 9ull * ptr[n_nodes];
    free(ptr); free(nbr);
    return nnz;
}

/* row_ptr per (:1092-1102); column fill either as the reference writes it
 * (neighbour-major across the node's three rows, :1109-1119: row 3n+d ends
 * up with neighbours d*k/3..(d+1)*k/3-1 each repeated three times) or the
 * solve pattern (every row of node n holds all 3*|nb(n)| columns, ascending). */
static void orc_pattern(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn, int as_reference,
                        uint32_t* row_ptr, uint32_t* col_idx) {
    uint32_t *ptr, *nbr;
    orc_node_neighbours(n_nodes, n_elems, conn, &ptr, &nbr);
    const uint32_t n_dofs = 3 * n_nodes;
    row_ptr[0] = 0;
    for (uint32_t n = 0; n < n_nodes; ++n) {
        uint32_t deg = ptr[n + 1] - ptr[n];
        for (int d = 0; d < 3; ++d) row_ptr[3 * n + d + 1] = row_ptr[3 * n + d] + 3 * deg;
    }
    (void)n_dofs;
    if (as_reference) {
        uint32_t w = 0;
        for (uint32_t n = 0; n < n_nodes; ++n)
            for (uint32_t k = ptr[n]; k < ptr[n + 1]; ++k)
                for (int ds = 0; ds < 3; ++ds)
                    for (int dn = 0; dn < 3; ++dn) col_idx[w++] = 3 * nbr[k] + (uint32_t)dn;
    } else {
        for (uint32_t n = 0; n < n_nodes; ++n)
            for (int d = 0; d < 3; ++d) {
                uint32_t w = row_ptr[3 * n + d];
                for (uint32_t k = ptr[n]; k < ptr[n + 1]; ++k)
                    for (int dn = 0; dn < 3; ++dn) col_idx[w++] = 3 * nbr[k] + (uint32_t)dn;
            }
    }
    free(ptr); free(nbr);
}

void orc_pattern_reference(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn,
                           uint32_t* row_ptr, uint32_t* col_idx) {
    orc_pattern(n_nodes, n_elems, conn, 1, row_ptr, col_idx);
}
void orc_pattern_solve(uint32_t n_nodes, uint32_t n_elems, const uint32_t* conn,
                       uint32_t* row_ptr, uint32_t* col_idx) {
    orc_pattern(n_nodes, n_elems, conn, 0, row_ptr, col_idx);
}

/* A4: element -> CSR slot map, slot[e][(i*3+di)*12 + j*3+dj].
 * Semantics of the reference's per-row hash map (:1141-1150, 1204-1211):
 * the LAST occurrence of a column in the row wins, a missing column is -1. */
void orc_slot_map(uint32_t n_dofs, uint32_t n_elems, const uint32_t* conn, const uint32_t* row_ptr,
                  const uint32_t* col_idx, int32_t* slot) {
    (void)n_dofs;
    for (uint32_t e = 0; e < n_elems; ++e) {
        const uint32_t* c = conn + 4 * (size_t)e;
        for (int i = 0; i < 4; ++i)
            for (int di = 0; di < 3; ++di) {
                uint32_t gi = 3 * c[i] + (uint32_t)di;
                for (int j = 0; j < 4; ++j)
                    for (int dj = 0; dj < 3; ++dj) {
                        uint32_t gj = 3 * c[j] + (uint32_t)dj;
                        int32_t found = -1;
                        for (uint32_t k = row_ptr[gi]; k < row_ptr[gi + 1]; ++k)
                            if (col_idx[k] == gj) found = (int32_t)k;
                        slot[144 * (size_t)e + (i * 3 + di) * 12 + j * 3 + dj] = found;
                    }
            }
    }
}

/* ------------------------------------------------------------------ */
/* A5-A8: element force and tangent                                    */
/* ------------------------------------------------------------------ */
/* cofactor inverse with the |det| < 1e-30 guard, FEM/adaptive_fem_engine.hpp:52-71 */
static void orc_inv3(const double A[9], double R[9]) {
    double det = A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) +
                 A[6] * (A[1] * A[5] - A[4] * A[2]);
    if (fabs(det) < 1e-30) {
        for (int q = 0; q < 9; ++q) R[q] = 0.0;
        R[0] = R[4] = R[8] = 1e30;
        return;
    }
    double s = 1.0 / det;
    R[0] = (A[4] * A[8] - A[7] * A[5]) * s;
    R[1] = -(A[1] * A[8] - A[7] * A[2]) * s;
    R[2] = (A[1] * A[5] - A[4] * A[2]) * s;
    R[3] = -(A[3] * A[8] - A[6] * A[5]) * s;
    R[4] = (A[0] * A[8] - A[6] * A[2]) * s;
    R[5] = -(A[0] * A[5] - A[3] * A[2]) * s;
    R[6] = (A[3] * A[7] - A[6] * A[4]) * s;
    R[7] = -(A[0] * A[7] - A[6] * A[1]) * s;
    R[8] = (A[0] * A[4] - A[3] * A[1]) * s;
}

static double orc_det3(const double A[9]) {
    return A[0] * (A[4] * A[8] - A[7] * A[5]) - A[3] * (A[1] * A[8] - A[7] * A[2]) +
           A[6] * (A[1] * A[5] - A[4] * A[2]);
}

/* Lame constants from (E, nu) exactly as the reference forms them (:81-82) */
void orc_lame(double E, double nu, double* mu, double* lam) {
    *mu = E / (2.0 * (1.0 + nu));
    *lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
}

/* Mandel stress of the compressible Neo-Hookean law (:79-129):
 * C = F^T F, S = mu (I - C^-1) + lam ln(max(J,0.01)) C^-1, M = C S. */
static void orc_mandel(const double F[9], double mu, double lam, double J, double sig[6]) {
    double C[9], Ci[9], S[9], M[9];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += F[k * 3 + a] * F[k * 3 + b];
            C[a * 3 + b] = s;
        }
    orc_inv3(C, Ci);
    double Js = J < 0.01 ? 0.01 : J;
    double lnJ = log(Js);
    for (int q = 0; q < 9; ++q) S[q] = mu * ((q % 4 == 0 ? 1.0 : 0.0) - Ci[q]) + lam * lnJ * Ci[q];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += C[a * 3 + k] * S[k * 3 + b];
            M[a * 3 + b] = s;
        }
    sig[0] = M[0];
    sig[1] = M[4];
    sig[2] = M[8];
    sig[3] = M[1] * ORC_SQRT2;
    sig[4] = M[2] * ORC_SQRT2;
    sig[5] = M[5] * ORC_SQRT2;
}

/* heuristic 6x6 Voigt tangent (:135-187) */
static void orc_tangent6(double mu, double lam, double nu, double J, double T[36]) {
    double Js = J < 0.01 ? 0.01 : J;
    double invJ = 1.0 / (Js + 1e-30);
    double lnJ = log(Js);
    for (int q = 0; q < 36; ++q) T[q] = 0.0;
    double bulk = lam + 2.0 * mu / 3.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) T[a * 6 + b] = (a == b) ? 2.0 * mu + bulk : bulk - 2.0 * mu / 3.0;
    T[3 * 6 + 3] = mu;
    T[4 * 6 + 4] = mu;
    T[5 * 6 + 5] = mu;
    double one_m = 1.0 - 2.0 * nu;
    double vol_f = (lam * invJ) / (one_m < 0.1 ? 0.1 : one_m);
    for (int a = 0; a < 3; ++a) T[a * 6 + a] += vol_f;
    double cross = -2.0 * lam * lnJ * invJ / 3.0;
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b)
            if (a != b) T[a * 6 + b] += cross;
}

/* Shape gradients, F and J of one tet.  Returns vol (0 => degenerate). */
static double orc_kinematics(const double x[12], const double u[12], double dN[4][3], double F[9],
                             double* Jdet) {
    double Jm[9], Ji[9];
    for (int d = 0; d < 3; ++d) {
        Jm[d * 3 + 0] = x[3 + d] - x[d];
        Jm[d * 3 + 1] = x[6 + d] - x[d];
        Jm[d * 3 + 2] = x[9 + d] - x[d];
    }
    orc_inv3(Jm, Ji);
    double vol = fabs(orc_det3(Jm)) / 6.0;
    if (vol < 1e-30) return 0.0;
    /* dN_a = J^-T dN_xi(a); dN_xi = (-1,-1,-1),(1,0,0),(0,1,0),(0,0,1) */
    for (int c = 0; c < 3; ++c) {
        dN[0][c] = -Ji[0 * 3 + c];
        dN[0][c] -= Ji[1 * 3 + c];
        dN[0][c] -= Ji[2 * 3 + c];
        dN[1][c] = Ji[0 * 3 + c];
        dN[2][c] = Ji[1 * 3 + c];
        dN[3][c] = Ji[2 * 3 + c];
    }
    double G[9];
    for (int a = 0; a < 3; ++a)
        for (int b = 0; b < 3; ++b) {
            double s = 0.0;
            for (int n = 0; n < 4; ++n) s += u[n * 3 + a] * dN[n][b];
            G[a * 3 + b] = s;
        }
    for (int q = 0; q < 9; ++q) F[q] = (q % 4 == 0) ? 1.0 + G[q] : G[q];
    *Jdet = orc_det3(F);
    return vol;
}

/* A5: 12x12 tangent and 12-vector internal force of one tet (:511-701).
 * mu, lam per element; nu enters only the volumetric tangent factor. */
void orc_element_lame(const double x[12], const double u[12], double mu, double lam, double nu,
                      double K[144], double f[12]) {
    double dN[4][3], F[9], J;
    double vol = orc_kinematics(x, u, dN, F, &J);
    if (vol == 0.0) {
        for (int q = 0; q < 144; ++q) K[q] = 0.0;
        for (int q = 0; q < 12; ++q) f[q] = 0.0;
        return;
    }
    double sig[6], T[36];
    orc_mandel(F, mu, lam, J, sig);
    orc_tangent6(mu, lam, nu, J, T);
    /* material part vol * B_a^T T B_b with the 6x3 Voigt B of each node */
    double B[4][18];
    for (int a = 0; a < 4; ++a) {
        double* b = B[a];
        for (int q = 0; q < 18; ++q) b[q] = 0.0;
        b[0 * 3 + 0] = dN[a][0]; b[1 * 3 + 1] = dN[a][1]; b[2 * 3 + 2] = dN[a][2];
        b[3 * 3 + 1] = dN[a][0]; b[3 * 3 + 0] = dN[a][1];
        b[4 * 3 + 2] = dN[a][0]; b[4 * 3 + 0] = dN[a][2];
        b[5 * 3 + 2] = dN[a][1]; b[5 * 3 + 1] = dN[a][2];
    }
    for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 4; ++c) {
            double TB[18];
            for (int r = 0; r < 6; ++r)
                for (int q = 0; q < 3; ++q) {
                    double s = 0.0;
                    for (int t = 0; t < 6; ++t) s += B[a][t * 3 + q] * T[r * 6 + t];
                    TB[r * 3 + q] = s;
                }
            for (int p = 0; p < 3; ++p)
                for (int q = 0; q < 3; ++q) {
                    double s = 0.0;
                    for (int r = 0; r < 6; ++r) s += TB[r * 3 + p] * B[c][r * 3 + q];
                    K[(a * 3 + p) * 12 + c * 3 + q] = vol * s;
                }
        }
    /* geometric part vol * (dN_a . sigma . dN_b) I (:649-692) */
    double S[9] = {sig[0],           sig[3] / ORC_SQRT2, sig[4] / ORC_SQRT2,
                   sig[3] / ORC_SQRT2, sig[1],           sig[5] / ORC_SQRT2,
                   sig[4] / ORC_SQRT2, sig[5] / ORC_SQRT2, sig[2]};
    for (int a = 0; a < 4; ++a)
        for (int c = 0; c < 4; ++c) {
            double g = 0.0;
            for (int al = 0; al < 3; ++al)
                for (int ga = 0; ga < 3; ++ga) g += dN[a][al] * S[al * 3 + ga] * dN[c][ga];
            for (int p = 0; p < 3; ++p) {
                for (int q = 0; q < 3; ++q) {
                    double add = (p == q) ? g : 0.0;
                    K[(a * 3 + p) * 12 + c * 3 + q] += vol * add;
                }
            }
        }
    /* internal force vol * M dN_a (:694-700) */
    for (int a = 0; a < 4; ++a) {
        f[a * 3 + 0] = 0.0 + vol * (dN[a][0] * sig[0] + dN[a][1] * sig[3] / ORC_SQRT2 +
                                    dN[a][2] * sig[4] / ORC_SQRT2);
        f[a * 3 + 1] = 0.0 + vol * (dN[a][1] * sig[1] + dN[a][0] * sig[3] / ORC_SQRT2 +
                                    dN[a][2] * sig[5] / ORC_SQRT2);
        f[a * 3 + 2] = 0.0 + vol * (dN[a][2] * sig[2] + dN[a][0] * sig[4] / ORC_SQRT2 +
                                    dN[a][1] * sig[5] / ORC_SQRT2);
    }
}

void orc_element(const double x[12], const double u[12], double E, double nu, double K[144],
                 double f[12]) {
    double mu, lam;
    orc_lame(E, nu, &mu, &lam);
    orc_element_lame(x, u, mu, lam, nu, K, f);
}

/* ------------------------------------------------------------------ */
/* A10/A11: global assembly in element order (1 thread semantics)     */
/* FEM/adaptive_fem_engine.hpp:1126-1233, 990-1059                     */
/* ------------------------------------------------------------------ */
static void orc_gather(const double* xyz, const double* u, const uint32_t* c, double x[12],
                       double ue[12]) {
    for (int a = 0; a < 4; ++a)
        for (int d = 0; d < 3; ++d) {
            x[a * 3 + d] = xyz[3 * (size_t)c[a] + d];
            ue[a * 3 + d] = u[3 * (size_t)c[a] + d];
        }
}

/* Material arrays: mu_e/lam_e per element (either may be the same scalar
 * repeated).  active[e] == 0 skips the element (stored volume < 1e-30,
 * :1169); NULL => all active.  K may be NULL (residual only). */
void orc_assemble(uint32_t n_nodes, uint32_t n_elems, const double* xyz, const uint32_t* conn,
                  const uint8_t* active, const double* mu_e, const double* lam_e, double nu,
                  const double* u, const int32_t* slot, uint64_t nnz, double* K, double* f_int) {
    const uint32_t n_dofs = 3 * n_nodes;
    if (K) memset(K, 0, sizeof(double) * nnz);
    memset(f_int, 0, sizeof(double) * n_dofs);
    double x[12], ue[12], Ke[144], fe[12];
    for (uint32_t e = 0; e < n_elems; ++e) {
        if (active && !active[e]) continue;
        const uint32_t* c = conn + 4 * (size_t)e;
        orc_gather(xyz, u, c, x, ue);
        orc_element_lame(x, ue, mu_e[e], lam_e[e], nu, Ke, fe);
        if (K) {
            const int32_t* s = slot + 144 * (size_t)e;
            for (int q = 0; q < 144; ++q)
                if (s[q] >= 0) K[s[q]] += Ke[q];
        }
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) f_int[3 * (size_t)c[a] + d] += fe[a * 3 + d];
    }
}

/* ------------------------------------------------------------------ */
/* A12: Dirichlet elimination, FEM/nonlinear_solver.hpp:329-334,388-396 */
/* ------------------------------------------------------------------ */
void orc_apply_bc(uint32_t n_dofs, const uint32_t* row_ptr, const uint32_t* col_idx, double* K,
                  double* R, const uint8_t* mask) {
    for (uint32_t i = 0; i < n_dofs; ++i) {
        if (R && mask[i]) R[i] = 0.0;
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            uint32_t j = col_idx[k];
            if (mask[i] || mask[j]) K[k] = (i == j) ? 1.0 : 0.0;
        }
    }
}

/* ------------------------------------------------------------------ */
/* A17: CSR SpMV in ascending slot order, FEM/fem_types.hpp:310-319    */
/* ------------------------------------------------------------------ */
void orc_spmv(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* val,
              const double* x, double* y) {
    for (uint32_t i = 0; i < n; ++i) {
        double s = 0.0;
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) s += val[k] * x[col_idx[k]];
        y[i] = s;
    }
}

/* ------------------------------------------------------------------ */
/* A13/A14: ILU(0).  Row-wise IKJ elimination in natural order.        */
/* The reference's Doolittle loop (FEM/adaptive_fem_engine.hpp:305-470) */
/* always picks rows in natural order and subtracts L(i,l)U(l,j) for   */
/* ascending l, which is the same operation sequence; pivots with      */
/* |u_ii| < 1e-12 are pushed by 1e-8 away from zero (:383-387).        */
/* Requires ascending, unique columns per row.                          */
/* Output: LU[k] holds L multipliers on strictly lower slots, U on     */
/* strictly upper slots, the matrix value on the diagonal slot (as the */
/* reference's U_val keeps it); diag[i] holds the pivots.              */
/* Returns the number of perturbed pivots.                             */
/* ------------------------------------------------------------------ */
int orc_ilu0(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* A,
             double* LU, double* diag) {
    int32_t* pos = (int32_t*)malloc(sizeof(int32_t) * n);
    for (uint32_t i = 0; i < n; ++i) pos[i] = -1;
    int perturbed = 0;
    memcpy(LU, A, sizeof(double) * row_ptr[n]);
    for (uint32_t i = 0; i < n; ++i) {
        uint32_t b = row_ptr[i], e = row_ptr[i + 1];
        for (uint32_t k = b; k < e; ++k) pos[col_idx[k]] = (int32_t)k;
        double u_ii = 0.0;
        int has_diag = 0;
        int32_t dslot = pos[i];
        if (dslot >= 0) { u_ii = A[dslot]; has_diag = 1; }
        for (uint32_t k = b; k < e; ++k) {
            uint32_t c = col_idx[k];
            if (c >= i) break;
            double l = LU[k] / diag[c];
            LU[k] = l;
            /* subtract l * U(c, j) for j > c present in row i */
            for (uint32_t m = row_ptr[c]; m < row_ptr[c + 1]; ++m) {
                uint32_t j = col_idx[m];
                if (j <= c) continue;
                /* the pivot accumulates U(c,i) even when (i,i) is not in
                 * row i's pattern (the reference looks U(c,i) up directly) */
                if (j == i) { u_ii -= l * LU[m]; continue; }
                int32_t t = pos[j];
                if (t < 0) continue;
                LU[t] -= l * LU[m];
            }
        }
        (void)has_diag;
        if (fabs(u_ii) < 1e-12) { u_ii += (u_ii >= 0 ? 1e-8 : -1e-8); ++perturbed; }
        diag[i] = u_ii;
        for (uint32_t k = b; k < e; ++k) pos[col_idx[k]] = -1;
    }
    free(pos);
    return perturbed;
}

/* A16: forward L z = r (unit lower), then U y = z with pivots (:473-504) */
void orc_ilu0_apply(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* LU,
                    const double* diag, const double* r, double* y, double* z_work) {
    double* z = z_work;
    for (uint32_t i = 0; i < n; ++i) {
        double s = r[i];
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            uint32_t c = col_idx[k];
            if (c < i) s -= LU[k] * z[c];
        }
        z[i] = s;
    }
    for (uint32_t ii = n; ii-- > 0;) {
        double s = z[ii];
        for (uint32_t k = row_ptr[ii]; k < row_ptr[ii + 1]; ++k) {
            uint32_t c = col_idx[k];
            if (c > ii) s -= LU[k] * y[c];
        }
        y[ii] = s / diag[ii];
    }
}

/* A15: true level sets. depth_L(i) = 1 + max depth_L(j), j < i in row i;
 * depth_U(i) = 1 + max depth_U(j), j > i.  Levels are the stable sort of
 * rows by depth.  Returns number of levels; ptr has (levels+1) entries. */
static uint32_t orc_levels_dir(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                               int upper, uint32_t* lvl_ptr, uint32_t* lvl_rows) {
    uint32_t* depth = (uint32_t*)malloc(sizeof(uint32_t) * n);
    uint32_t maxd = 0;
    for (uint32_t t = 0; t < n; ++t) {
        uint32_t i = upper ? n - 1 - t : t;
        uint32_t d = 0;
        for (uint32_t k = row_ptr[i]; k < row_ptr[i + 1]; ++k) {
            uint32_t c = col_idx[k];
            if ((!upper && c < i) || (upper && c > i))
                if (depth[c] + 1 > d) d = depth[c] + 1;
        }
        depth[i] = d;
        if (d > maxd) maxd = d;
    }
    uint32_t nl = n ? maxd + 1 : 0;
    memset(lvl_ptr, 0, sizeof(uint32_t) * (nl + 1));
    for (uint32_t i = 0; i < n; ++i) lvl_ptr[depth[i] + 1]++;
    for (uint32_t l = 0; l < nl; ++l) lvl_ptr[l + 1] += lvl_ptr[l];
    uint32_t* fill = (uint32_t*)calloc(nl + 1, sizeof(uint32_t));
    for (uint32_t i = 0; i < n; ++i) lvl_rows[lvl_ptr[depth[i]] + fill[depth[i]]++] = i;
    free(fill);
    free(depth);
    return nl;
}

/* lvl_ptr arrays need n+1 entries of room */
void orc_levels(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, uint32_t* fwd_ptr,
                uint32_t* fwd_rows, uint32_t* bwd_ptr, uint32_t* bwd_rows, uint32_t* n_fwd,
                uint32_t* n_bwd) {
    *n_fwd = orc_levels_dir(n, row_ptr, col_idx, 0, fwd_ptr, fwd_rows);
    *n_bwd = orc_levels_dir(n, row_ptr, col_idx, 1, bwd_ptr, bwd_rows);
}

/* ------------------------------------------------------------------ */
/* A18: PCG with ILU(0), FEM/adaptive_fem_engine.hpp:1283-1341         */
/* Same stop tests: early exit when ||b - A x0|| < tol*1e-3, breakdown */
/* when |p.Ap| < 1e-60, convergence when sqrt(rz/b.b) < tol.           */
/* The factorization is computed on entry as in the reference.         */
/* Returns iterations (max_iter when not converged).                   */
/* ------------------------------------------------------------------ */
/* Copy of a CSR matrix with each row's columns sorted ascending (the
 * reference sorts its L/U patterns, :256-258, while SpMV keeps the given
 * order).  Returns 1 and fills cs and vs when a copy was needed. */
static int orc_sorted(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx,
                      const double* val, uint32_t** cs, double** vs) {
    int sorted = 1;
    for (uint32_t i = 0; i < n && sorted; ++i)
        for (uint32_t k = row_ptr[i] + 1; k < row_ptr[i + 1]; ++k)
            if (col_idx[k] <= col_idx[k - 1]) { sorted = 0; break; }
    if (sorted) return 0;
    size_t nnz = row_ptr[n];
    uint32_t* c = (uint32_t*)malloc(sizeof(uint32_t) * nnz + 4);
    double* v = (double*)malloc(sizeof(double) * nnz + 8);
    memcpy(c, col_idx, sizeof(uint32_t) * nnz);
    memcpy(v, val, sizeof(double) * nnz);
    for (uint32_t i = 0; i < n; ++i)
        for (uint32_t x = row_ptr[i] + 1; x < row_ptr[i + 1]; ++x) {
            uint32_t cc = c[x];
            double vv = v[x];
            uint32_t y = x;
            while (y > row_ptr[i] && c[y - 1] > cc) { c[y] = c[y - 1]; v[y] = v[y - 1]; --y; }
            c[y] = cc;
            v[y] = vv;
        }
    *cs = c;
    *vs = v;
    return 1;
}

int orc_pcg_ilu0(uint32_t n, const uint32_t* row_ptr, const uint32_t* col_idx, const double* A,
                 const double* b, double* x, double tol, int max_iter, double* relres_out) {
    uint32_t* cs = NULL;
    double* As = NULL;
    int own = orc_sorted(n, row_ptr, col_idx, A, &cs, &As);
    const uint32_t* ci = own ? cs : col_idx;
    double* LU = (double*)malloc(sizeof(double) * row_ptr[n]);
    double* diag = (double*)malloc(sizeof(double) * n);
    double* r = (double*)malloc(sizeof(double) * n);
    double* p = (double*)malloc(sizeof(double) * n);
    double* Ap = (double*)malloc(sizeof(double) * n);
    double* z = (double*)malloc(sizeof(double) * n);
    double* w = (double*)malloc(sizeof(double) * n);
    orc_ilu0(n, row_ptr, ci, own ? As : A, LU, diag);
    int it_out = max_iter;
    double relres = 0.0;
    orc_spmv(n, row_ptr, col_idx, A, x, Ap);
    double rr = 0.0;
    for (uint32_t i = 0; i < n; ++i) { r[i] = b[i] - Ap[i]; rr += r[i] * r[i]; }
    if (sqrt(rr) < tol * 1e-3) { it_out = 0; goto done; }
    orc_ilu0_apply(n, row_ptr, ci, LU, diag, r, z, w);
    double rz = 0.0;
    for (uint32_t i = 0; i < n; ++i) { p[i] = z[i]; rz += r[i] * z[i]; }
    double bb = 0.0;
    for (uint32_t i = 0; i < n; ++i) bb += b[i] * b[i];
    for (int it = 0; it < max_iter; ++it) {
        orc_spmv(n, row_ptr, col_idx, A, p, Ap);
        double pAp = 0.0;
        for (uint32_t i = 0; i < n; ++i) pAp += p[i] * Ap[i];
        if (fabs(pAp) < 1e-60) break;
        double alpha = rz / pAp;
        for (uint32_t i = 0; i < n; ++i) { x[i] += alpha * p[i]; r[i] -= alpha * Ap[i]; }
        orc_ilu0_apply(n, row_ptr, ci, LU, diag, r, z, w);
        double rz_new = 0.0;
        for (uint32_t i = 0; i < n; ++i) rz_new += r[i] * z[i];
        relres = sqrt(rz_new / (bb > 1e-300 ? bb : 1e-300));
        if (relres < tol) { it_out = it + 1; goto done; }
        double beta = rz_new / rz;
        for (uint32_t i = 0; i < n; ++i) p[i] = z[i] + beta * p[i];
        rz = rz_new;
    }
done:
    if (relres_out) *relres_out = relres;
    free(LU); free(diag); free(r); free(p); free(Ap); free(z); free(w);
    if (own) { free(cs); free(As); }
    return it_out;
}

/* ------------------------------------------------------------------ */
/* A19: Newton with Dirichlet elimination and load stepping            */
/* Contract (the reference's Newton, FEM/adaptive_fem_engine.hpp:2476-  */
/* 2592, with elimination BCs as FEM/nonlinear_solver.hpp:329-334,     */
/* 388-396, driven by prescribed displacements):                       */
/*  load step s, level f = s/S, prescribed increment v = f*val - u on  */
/*  the constrained DOFs (0 elsewhere):                                */
/*  predictor (when v != 0): K, f_int at u without elimination;        */
/*    R = -f_int - K v on free DOFs, 0 on constrained; r0 = ||R||;     */
/*    eliminate; du = PCG(K, R); u_free += du; u_c = f*val.            */
/*  Newton: assemble, eliminate, R = -f_int (0 on constrained);        */
/*    stop when ||R|| < rtol * r0 (r0 = first ||R|| if no predictor);  */
/*    du = PCG-ILU(0)(K, R) to inner_tol; u += du.                     */
/* The predictor spreads the boundary increment through the body       */
/* (a linearized lifting); without it a full increment on the top face */
/* puts a strain of u_z/h into the top element layer and the Newton    */
/* iteration with the reference's tangent diverges on fine meshes.    */
/* Newton counts include the predictor solve.                          */
/* Returns 0 on convergence of every step, 1 otherwise.                */
/* ------------------------------------------------------------------ */
/* Free-DOF 2-norm of R = -f (constrained entries zero) */
static double orc_free_norm(uint32_t n, const double* f, const uint8_t* mask) {
    double s = 0.0;
    for (uint32_t i = 0; i < n; ++i)
        if (!mask[i]) s += f[i] * f[i];
    return sqrt(s);
}

/* Newton load steps first_step..last_step of an n_steps path, with the
 * options of the GPU path's fm_newton_config:
 *  - each load step starts with the linearized Dirichlet predictor
 *    K_ff du_f = -f_f - K_fc v_c (v: the prescribed increment), solved to
 *    predictor_tol (<= 0: inner_tol);
 *  - Newton iterations: assemble, eliminate, R = -f, stop at
 *    ||R|| < rtol ||R_0||, PCG to inner_tol, u += alpha du;
 *  - line_search > 0: alpha from armijo_line_search_true
 *    (FEM/adaptive_fem_engine.hpp:933-985): alpha = 1, 1/2, ... accepted
 *    when ||R(u + alpha du)|| <= (1 - ls_c alpha) ||R(u)|| + 1e-14 (residual
 *    re-assembled at each trial), 2^-line_search when none is accepted;
 *  - the reference's divergence test (:2561-2572), from the fourth
 *    iteration of a step on: rate = ||R|| / ||R_prev|| > diverge_rate counts
 *    a slow iteration; stop when more than diverge_count were slow or
 *    ||R|| > diverge_growth ||R_prev|| (<= 0 disables each half).
 * Returns 0, 1 (a step hit max_newton) or 2 (the divergence test stopped a
 * step; the remaining steps are not run).  alpha_hist (nullable) receives the
 * step length of every Newton iteration (predictor excluded), up to alpha_cap. */
int orc_newton_ex(uint32_t n_nodes, uint32_t n_elems, const double* xyz, const uint32_t* conn,
                  const uint8_t* active, const double* mu_e, const double* lam_e, double nu,
                  const uint32_t* row_ptr, const uint32_t* col_idx, const int32_t* slot,
                  const uint8_t* mask, const double* bc_value, int first_step, int last_step,
                  int n_steps, double rtol, double inner_tol, double predictor_tol,
                  int max_newton, int max_pcg, int line_search, double ls_c,
                  double diverge_rate, int diverge_count, double diverge_growth, double* u,
                  int* newton_per_step, int* pcg_per_step, double* alpha_hist, int alpha_cap,
                  int* n_alpha) {
    const uint32_t n = 3 * n_nodes;
    const uint64_t nnz = row_ptr[n];
    double* K = (double*)malloc(sizeof(double) * nnz);
    double* f = (double*)malloc(sizeof(double) * n);
    double* R = (double*)malloc(sizeof(double) * n);
    double* du = (double*)malloc(sizeof(double) * n);
    double* v = (double*)malloc(sizeof(double) * n);
    double* ut = (double*)malloc(sizeof(double) * n);
    int status = 0, na = 0;
    const double ptol = predictor_tol > 0.0 ? predictor_tol : inner_tol;
    for (int s = first_step; s <= last_step && status != 2; ++s) {
        double frac = (double)s / (double)n_steps;
        double r0 = 0.0, r_prev = 0.0;
        int it = 0, pcg_total = 0, conv = 0, have_r0 = 0, slow = 0;
        int any = 0;
        for (uint32_t i = 0; i < n; ++i) {
            v[i] = mask[i] ? frac * bc_value[i] - u[i] : 0.0;
            if (v[i] != 0.0) any = 1;
        }
        if (any) {
            orc_assemble(n_nodes, n_elems, xyz, conn, active, mu_e, lam_e, nu, u, slot, nnz, K, f);
            orc_spmv(n, row_ptr, col_idx, K, v, R);
            for (uint32_t i = 0; i < n; ++i) R[i] = mask[i] ? 0.0 : -f[i] - R[i];
            orc_apply_bc(n, row_ptr, col_idx, K, NULL, mask);
            for (uint32_t i = 0; i < n; ++i) r0 += R[i] * R[i];
            r0 = sqrt(r0);
            have_r0 = 1;
            memset(du, 0, sizeof(double) * n);
            pcg_total += orc_pcg_ilu0(n, row_ptr, col_idx, K, R, du, ptol, max_pcg, NULL);
            for (uint32_t i = 0; i < n; ++i) u[i] = mask[i] ? frac * bc_value[i] : u[i] + du[i];
            r_prev = r0;
            it = 1;
        }
        for (; it < max_newton; ++it) {
            orc_assemble(n_nodes, n_elems, xyz, conn, active, mu_e, lam_e, nu, u, slot, nnz, K, f);
            for (uint32_t i = 0; i < n; ++i) R[i] = -f[i];
            orc_apply_bc(n, row_ptr, col_idx, K, R, mask);
            double rn = 0.0;
            for (uint32_t i = 0; i < n; ++i) rn += R[i] * R[i];
            rn = sqrt(rn);
            if (!have_r0) { r0 = rn; have_r0 = 1; }
            if (rn == 0.0 || rn < rtol * r0) { conv = 1; break; }
            if (it > 2) {
                const double rate = rn / (r_prev > 1e-30 ? r_prev : 1e-30);
                if (diverge_rate > 0.0 && rate > diverge_rate) ++slow;
                if ((diverge_rate > 0.0 && slow > diverge_count) ||
                    (diverge_growth > 0.0 && rn > r_prev * diverge_growth)) {
                    status = 2;
                    break;
                }
            }
            memset(du, 0, sizeof(double) * n);
            pcg_total += orc_pcg_ilu0(n, row_ptr, col_idx, K, R, du, inner_tol, max_pcg, NULL);
            double alpha = 1.0;
            if (line_search > 0) {
                for (int bt = 0; bt < line_search; ++bt) {
                    for (uint32_t i = 0; i < n; ++i) ut[i] = u[i] + alpha * du[i];
                    orc_assemble(n_nodes, n_elems, xyz, conn, active, mu_e, lam_e, nu, ut, NULL, 0,
                                 NULL, f);
                    if (orc_free_norm(n, f, mask) <= (1.0 - ls_c * alpha) * rn + 1e-14) break;
                    alpha *= 0.5;
                }
            }
            for (uint32_t i = 0; i < n; ++i) u[i] += alpha * du[i];
            if (alpha_hist && na < alpha_cap) alpha_hist[na] = alpha;
            ++na;
            r_prev = rn;
        }
        if (!conv && status != 2) status = 1;
        if (newton_per_step) newton_per_step[s - first_step] = it;
        if (pcg_per_step) pcg_per_step[s - first_step] = pcg_total;
    }
    if (n_alpha) *n_alpha = na;
    free(K); free(f); free(R); free(du); free(v); free(ut);
    return status;
}

int orc_newton(uint32_t n_nodes, uint32_t n_elems, const double* xyz, const uint32_t* conn,
               const uint8_t* active, const double* mu_e, const double* lam_e, double nu,
               const uint32_t* row_ptr, const uint32_t* col_idx, const int32_t* slot,
               const uint8_t* mask, const double* bc_value, int n_steps, double rtol,
               double inner_tol, int max_newton, int max_pcg, double* u, int* newton_per_step,
               int* pcg_per_step) {
    return orc_newton_ex(n_nodes, n_elems, xyz, conn, active, mu_e, lam_e, nu, row_ptr, col_idx,
                         slot, mask, bc_value, 1, n_steps, n_steps, rtol, inner_tol, 0.0,
                         max_newton, max_pcg, 0, 0.0, 0.0, 0, 0.0, u, newton_per_step,
                         pcg_per_step, NULL, 0, NULL);
}

/* ------------------------------------------------------------------ */
/* A9/A21: exact Jacobian of the element force and the adjoint.        */
/* No reference code exists; derived from f_a = vol M dN_a with        */
/* M = C S = mu (C - I) + lam ln(max(J,0.01)) I:                       */
/*   dM/du_b,j : mu [ (g_b)_i F_jk + F_ji (g_b)_k ] + lam (F^-T g_b)_j d_ik */
/* (the lam term vanishes while J < 0.01).                             */
/* ------------------------------------------------------------------ */
/* out_a = vol * dM g_a for direction v (forward) */
static void orc_elem_jvp(const double dN[4][3], const double F[9], double J, double vol, double mu,
                         double lam, const double v[12], double out[12]) {
    double V[9];
    for (int a = 0; a < 3; ++a)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int b = 0; b < 4; ++b) s += v[b * 3 + a] * dN[b][k];
            V[a * 3 + k] = s;
        }
    double dC[9];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int m = 0; m < 3; ++m) s += V[m * 3 + i] * F[m * 3 + k] + F[m * 3 + i] * V[m * 3 + k];
            dC[i * 3 + k] = s;
        }
    double dlnJ = 0.0;
    if (J >= 0.01) {
        double Fi[9];
        orc_inv3(F, Fi);
        for (int k = 0; k < 3; ++k)
            for (int m = 0; m < 3; ++m) dlnJ += Fi[k * 3 + m] * V[m * 3 + k];
    }
    for (int a = 0; a < 4; ++a)
        for (int i = 0; i < 3; ++i) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k)
                s += (mu * dC[i * 3 + k] + (i == k ? lam * dlnJ : 0.0)) * dN[a][k];
            out[a * 3 + i] = vol * s;
        }
}

/* out_b = vol * [mu F (L + L^T) + lam tr(L) F^-T] g_b, L = sum_a lam_a (x) g_a */
static void orc_elem_vjp(const double dN[4][3], const double F[9], double J, double vol, double mu,
                         double lam, const double w[12], double out[12], double Lg[9]) {
    double L[9];
    for (int i = 0; i < 3; ++i)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int a = 0; a < 4; ++a) s += w[a * 3 + i] * dN[a][k];
            L[i * 3 + k] = s;
        }
    if (Lg) memcpy(Lg, L, sizeof(L));
    double Q[9];
    for (int j = 0; j < 3; ++j)
        for (int k = 0; k < 3; ++k) {
            double s = 0.0;
            for (int m = 0; m < 3; ++m) s += F[j * 3 + m] * (L[m * 3 + k] + L[k * 3 + m]);
            Q[j * 3 + k] = mu * s;
        }
    if (J >= 0.01) {
        double Fi[9];
        orc_inv3(F, Fi);
        double tr = L[0] + L[4] + L[8];
        for (int j = 0; j < 3; ++j)
            for (int k = 0; k < 3; ++k) Q[j * 3 + k] += lam * tr * Fi[k * 3 + j];
    }
    for (int b = 0; b < 4; ++b)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += Q[j * 3 + k] * dN[b][k];
            out[b * 3 + j] = vol * s;
        }
}

/* y = K_exact v (transpose=0) or K_exact^T v (transpose=1), matrix-free */
void orc_exact_apply(uint32_t n_nodes, uint32_t n_elems, const double* xyz, const uint32_t* conn,
                     const uint8_t* active, const double* mu_e, const double* lam_e,
                     const double* u, const double* v, double* y, int transpose) {
    memset(y, 0, sizeof(double) * 3 * (size_t)n_nodes);
    double x[12], ue[12], ve[12], dN[4][3], F[9], J, out[12];
    for (uint32_t e = 0; e < n_elems; ++e) {
        if (active && !active[e]) continue;
        const uint32_t* c = conn + 4 * (size_t)e;
        orc_gather(xyz, u, c, x, ue);
        double vol = orc_kinematics(x, ue, dN, F, &J);
        if (vol == 0.0) continue;
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) ve[a * 3 + d] = v[3 * (size_t)c[a] + d];
        if (transpose) orc_elem_vjp(dN, F, J, vol, mu_e[e], lam_e[e], ve, out, NULL);
        else orc_elem_jvp(dN, F, J, vol, mu_e[e], lam_e[e], ve, out);
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) y[3 * (size_t)c[a] + d] += out[a * 3 + d];
    }
}

/* Per-element parameter gradients from an adjoint vector w:
 * dL/dmu_e = -vol (C - I) : L_e,  dL/dlam_e = -vol ln(max(J,.01)) tr(L_e). */
void orc_param_grads(uint32_t n_elems, const double* xyz, const uint32_t* conn,
                     const uint8_t* active, const double* u, const double* w, double* g_mu,
                     double* g_lam) {
    double x[12], ue[12], we[12], dN[4][3], F[9], J, L[9];
    for (uint32_t e = 0; e < n_elems; ++e) {
        g_mu[e] = 0.0;
        g_lam[e] = 0.0;
        if (active && !active[e]) continue;
        const uint32_t* c = conn + 4 * (size_t)e;
        orc_gather(xyz, u, c, x, ue);
        double vol = orc_kinematics(x, ue, dN, F, &J);
        if (vol == 0.0) continue;
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) we[a * 3 + d] = w[3 * (size_t)c[a] + d];
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) {
                double s = 0.0;
                for (int a = 0; a < 4; ++a) s += we[a * 3 + i] * dN[a][k];
                L[i * 3 + k] = s;
            }
        double C[9];
        for (int i = 0; i < 3; ++i)
            for (int k = 0; k < 3; ++k) {
                double s = 0.0;
                for (int m = 0; m < 3; ++m) s += F[m * 3 + i] * F[m * 3 + k];
                C[i * 3 + k] = s;
            }
        double cm = 0.0;
        for (int q = 0; q < 9; ++q) cm += (C[q] - (q % 4 == 0 ? 1.0 : 0.0)) * L[q];
        double Js = J < 0.01 ? 0.01 : J;
        g_mu[e] = -vol * cm;
        g_lam[e] = -vol * log(Js) * (L[0] + L[4] + L[8]);
    }
}

/* Adjoint solve K_exact^T w = g on the free DOFs by defect correction with
 * the (symmetric) reference tangent K_t, whose eliminated CSR values are
 * given: w <- w + PCG(K_t, g - K_exact^T w).  Constrained DOFs stay 0.
 * Returns the number of correction sweeps (negative if not converged). */
int orc_adjoint(uint32_t n_nodes, uint32_t n_elems, const double* xyz, const uint32_t* conn,
                const uint8_t* active, const double* mu_e, const double* lam_e,
                const uint32_t* row_ptr, const uint32_t* col_idx, const double* Kt,
                const uint8_t* mask, const double* u, const double* g, double tol, double inner_tol,
                int max_sweeps, int max_pcg, double* w) {
    const uint32_t n = 3 * n_nodes;
    double* res = (double*)malloc(sizeof(double) * n);
    double* KTw = (double*)malloc(sizeof(double) * n);
    double* dw = (double*)malloc(sizeof(double) * n);
    memset(w, 0, sizeof(double) * n);
    double gn = 0.0;
    for (uint32_t i = 0; i < n; ++i)
        if (!mask[i]) gn += g[i] * g[i];
    gn = sqrt(gn);
    int sweep, ok = 0;
    for (sweep = 0; sweep < max_sweeps; ++sweep) {
        orc_exact_apply(n_nodes, n_elems, xyz, conn, active, mu_e, lam_e, u, w, KTw, 1);
        double rn = 0.0;
        for (uint32_t i = 0; i < n; ++i) {
            res[i] = mask[i] ? 0.0 : g[i] - KTw[i];
            rn += res[i] * res[i];
        }
        if (sqrt(rn) <= tol * gn) { ok = 1; break; }
        memset(dw, 0, sizeof(double) * n);
        orc_pcg_ilu0(n, row_ptr, col_idx, Kt, res, dw, inner_tol, max_pcg, NULL);
        for (uint32_t i = 0; i < n; ++i)
            if (!mask[i]) w[i] += dw[i];
    }
    free(res); free(KTw); free(dw);
    return ok ? sweep : -sweep - 1;
}

/* 2-D 5-point Poisson problem of the reference's validation runner
 * (TESTS/external_validation_runner.cpp:65-124): rows in (i,j) order, each
 * row lists the diagonal first, then (i-1,j), (i+1,j), (i,j-1), (i,j+1);
 * b = A x_exact with x_exact = sin(pi x) sin(pi y).  Caller sizes arrays
 * for 5*g*g entries; returns nnz. */
uint32_t orc_poisson(uint32_t g, uint32_t* row_ptr, uint32_t* col_idx, double* val, double* b,
                     double* x_exact) {
    const double h = 1.0 / (double)(g + 1);
    const double ih2 = 1.0 / (h * h);
    const double pi = 3.14159265358979323846;
    for (uint32_t i = 0; i < g; ++i) {
        double xx = (double)(i + 1) * h;
        for (uint32_t j = 0; j < g; ++j) {
            double yy = (double)(j + 1) * h;
            x_exact[i * g + j] = sin(pi * xx) * sin(pi * yy);
        }
    }
    uint32_t w = 0;
    for (uint32_t i = 0; i < g; ++i)
        for (uint32_t j = 0; j < g; ++j) {
            uint32_t row = i * g + j;
            row_ptr[row] = w;
            col_idx[w] = row; val[w++] = 4.0 * ih2;
            if (i > 0) { col_idx[w] = (i - 1) * g + j; val[w++] = -ih2; }
            if (i + 1 < g) { col_idx[w] = (i + 1) * g + j; val[w++] = -ih2; }
            if (j > 0) { col_idx[w] = i * g + j - 1; val[w++] = -ih2; }
            if (j + 1 < g) { col_idx[w] = i * g + j + 1; val[w++] = -ih2; }
        }
    row_ptr[g * g] = w;
    orc_spmv(g * g, row_ptr, col_idx, val, x_exact, b);
    return w;
}

/* ------------------------------------------------------------------ */
/* Element state update: update_element_states_rigorous               */
/* (FEM/adaptive_fem_engine.hpp:2716-2794) with the SL(3) retraction  */
/* of CORE/lie_operator.cpp (exp :95-152, Denman-Beavers square root  */
/* :164-184, log :200-268, retraction :300-311), restated on its      */
/* column-major Matrix3x3 data layout (a[c*3 + r]).                   */
/* ------------------------------------------------------------------ */
typedef struct { double a[9]; } orc_m3;

static orc_m3 m3_ident(void) { orc_m3 r = {{1, 0, 0, 0, 1, 0, 0, 0, 1}}; return r; }
static orc_m3 m3_zero(void) { orc_m3 r = {{0, 0, 0, 0, 0, 0, 0, 0, 0}}; return r; }
static orc_m3 m3_add(orc_m3 A, orc_m3 B) { for (int i = 0; i < 9; ++i) A.a[i] = A.a[i] + B.a[i]; return A; }
static orc_m3 m3_sub(orc_m3 A, orc_m3 B) { for (int i = 0; i < 9; ++i) A.a[i] = A.a[i] - B.a[i]; return A; }
static orc_m3 m3_scale(orc_m3 A, double s) { for (int i = 0; i < 9; ++i) A.a[i] = A.a[i] * s; return A; }
static orc_m3 m3_mul(orc_m3 A, orc_m3 B) {
    orc_m3 C;
    for (int c = 0; c < 3; ++c)
        for (int r = 0; r < 3; ++r)
            C.a[3 * c + r] = A.a[r] * B.a[3 * c] + A.a[3 + r] * B.a[3 * c + 1] + A.a[6 + r] * B.a[3 * c + 2];
    return C;
}
static double m3_trace(orc_m3 A) { return A.a[0] + A.a[4] + A.a[8]; }
static double m3_frob(orc_m3 A) {
    double s = 0.0;
    for (int i = 0; i < 9; ++i) s += A.a[i] * A.a[i];
    return sqrt(s);
}
static double m3_inf(orc_m3 A) {
    double m = 0.0;
    for (int r = 0; r < 3; ++r) {
        double t = fabs(A.a[r]) + fabs(A.a[3 + r]) + fabs(A.a[6 + r]);
        if (t > m) m = t;
    }
    return m;
}
static double m3_one(orc_m3 A) {
    double m = 0.0;
    for (int c = 0; c < 3; ++c) {
        double t = fabs(A.a[3 * c]) + fabs(A.a[3 * c + 1]) + fabs(A.a[3 * c + 2]);
        if (t > m) m = t;
    }
    return m;
}
static double m3_det(orc_m3 A) {
    return A.a[0] * (A.a[4] * A.a[8] - A.a[7] * A.a[5]) - A.a[3] * (A.a[1] * A.a[8] - A.a[7] * A.a[2]) +
           A.a[6] * (A.a[1] * A.a[5] - A.a[4] * A.a[2]);
}
static orc_m3 m3_inv(orc_m3 A) {
    const double a00 = A.a[0], a10 = A.a[1], a20 = A.a[2];
    const double a01 = A.a[3], a11 = A.a[4], a21 = A.a[5];
    const double a02 = A.a[6], a12 = A.a[7], a22 = A.a[8];
    const double c00 = a11 * a22 - a21 * a12, c10 = -(a01 * a22 - a21 * a02), c20 = a01 * a12 - a11 * a02;
    const double c01 = -(a10 * a22 - a20 * a12), c11 = a00 * a22 - a20 * a02, c21 = -(a00 * a12 - a10 * a02);
    const double c02 = a10 * a21 - a20 * a11, c12 = -(a00 * a21 - a20 * a01), c22 = a00 * a11 - a10 * a01;
    const double d = a00 * c00 + a10 * c10 + a20 * c20;
    if (fabs(d) < 1.0e-15) return m3_ident();
    const double id = 1.0 / d;
    orc_m3 r = {{c00 * id, c01 * id, c02 * id, c10 * id, c11 * id, c12 * id, c20 * id, c21 * id, c22 * id}};
    return r;
}
static double m3_cond(orc_m3 A) {
    if (fabs(m3_det(A)) < 1.0e-15) return 1.0e18;
    double k = m3_one(A) * m3_one(m3_inv(A));
    return k < 1.0e18 ? k : 1.0e18;
}
static orc_m3 m3_expm(orc_m3 A) {
    const double b1 = 0.5, b2 = 0.1, b3 = 1.0 / 120.0, theta3 = 1.495585217958292;
    const double nrm = m3_inf(A);
    if (!isfinite(nrm)) return m3_ident();
    int s = 0;
    if (nrm > theta3) s = (int)ceil(log2(nrm / theta3));
    if (m3_cond(A) > 1.0e8 && s < 8) ++s;
    const double sc = 1.0 / (double)(1LL << s);
    const orc_m3 X = m3_scale(A, sc), X2 = m3_mul(X, X), X3 = m3_mul(X2, X), I = m3_ident();
    const orc_m3 P = m3_add(m3_add(I, m3_scale(X, b1)), m3_add(m3_scale(X2, b2), m3_scale(X3, b3)));
    const orc_m3 Q = m3_add(m3_add(I, m3_scale(X, -b1)), m3_add(m3_scale(X2, b2), m3_scale(X3, -b3)));
    orc_m3 R = m3_mul(m3_inv(Q), P);
    for (int i = 0; i < s; ++i) R = m3_mul(R, R);
    const double dR = m3_det(R), target = exp(m3_trace(A));
    if (isfinite(dR) && isfinite(target) && dR > 1.0e-300 && target > 1.0e-300)
        R = m3_scale(R, cbrt(target / dR));
    return R;
}
static orc_m3 m3_sqrt_db(orc_m3 A) {
    orc_m3 Y = A, Z = m3_ident();
    for (int it = 0; it < 20; ++it) {
        if (m3_frob(m3_sub(m3_mul(Y, Y), A)) < 4.0e-16) break;
        const orc_m3 Yi = m3_inv(Y), Zi = m3_inv(Z);
        const orc_m3 Yn = m3_scale(m3_add(Y, Zi), 0.5), Zn = m3_scale(m3_add(Z, Yi), 0.5);
        Y = Yn;
        Z = Zn;
    }
    return Y;
}
static orc_m3 m3_logm(orc_m3 A) {
    double fs = 0.0;
    for (int i = 0; i < 9; ++i) fs += A.a[i] * A.a[i];
    if (!isfinite(fs)) return m3_zero();
    const orc_m3 I = m3_ident();
    {
        const orc_m3 E = m3_sub(A, I);
        if (m3_inf(E) < 1.0e-7) {
            const orc_m3 E2 = m3_mul(E, E), E3 = m3_mul(E2, E);
            return m3_add(m3_sub(E, m3_scale(E2, 0.5)), m3_scale(E3, 1.0 / 3.0));
        }
    }
    orc_m3 B = A;
    int roots = 0;
    for (int k = 0; k < 16; ++k) {
        if (m3_inf(m3_sub(B, I)) < 0.125) break;
        B = m3_sqrt_db(B);
        ++roots;
    }
    const orc_m3 Z = m3_mul(m3_sub(B, I), m3_inv(m3_add(B, I))), Z2 = m3_mul(Z, Z);
    orc_m3 Zp = Z, sum = Z;
    for (int k = 1; k <= 32; ++k) {
        Zp = m3_mul(Zp, Z2);
        sum = m3_add(sum, m3_scale(Zp, 1.0 / (double)(2 * k + 1)));
    }
    orc_m3 L = m3_scale(m3_scale(sum, 2.0), (double)(1LL << roots));
    orc_m3 best = L;
    double best_rel = INFINITY;
    const double fa = m3_frob(A), denom = fa > 1.0e-30 ? fa : 1.0e-30;
    for (int it = 0; it < 4; ++it) {
        const orc_m3 eL = m3_expm(L), res = m3_sub(A, eL);
        const double rel = m3_frob(res) / denom;
        if (isfinite(rel) && rel < best_rel) { best_rel = rel; best = L; }
        if (rel < 1.0e-12) break;
        const orc_m3 corr = m3_mul(res, m3_inv(eL));
        const double cn = m3_frob(corr);
        if (!isfinite(cn) || cn > 0.25) break;
        L = m3_add(L, corr);
    }
    return best;
}

/* sl3_retraction(G, 0): exp(log G) rescaled to det 1 */
void orc_sl3_retraction(const double G[9], double out[9]) {
    orc_m3 g;
    memcpy(g.a, G, sizeof g.a);
    orc_m3 R = m3_expm(m3_add(m3_logm(g), m3_zero()));
    const double d = m3_det(R);
    if (fabs(d) > 1.0e-15) R = m3_scale(R, 1.0 / cbrt(d));
    memcpy(out, R.a, sizeof R.a);
}

/* neo_hookean_response (:79-129) with a defined J */
void orc_nh_response(const double F[9], double mu, double lam, double J, double sig[6]) {
    double C[9], Ci[9], S[9], M[9];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += F[k * 3 + i] * F[k * 3 + j];
            C[i * 3 + j] = s;
        }
    orc_inv3(C, Ci);
    const double lnJ = log(J < 0.01 ? 0.01 : J);
    for (int i = 0; i < 9; ++i) S[i] = mu * ((i % 4 == 0 ? 1.0 : 0.0) - Ci[i]) + lam * lnJ * Ci[i];
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0.0;
            for (int k = 0; k < 3; ++k) s += C[i * 3 + k] * S[k * 3 + j];
            M[i * 3 + j] = s;
        }
    sig[0] = M[0];
    sig[1] = M[4];
    sig[2] = M[8];
    sig[3] = M[1] * ORC_SQRT2;
    sig[4] = M[2] * ORC_SQRT2;
    sig[5] = M[5] * ORC_SQRT2;
}

/* The update of every element's state at displacement u: F_sl3 (9 per tet)
 * and stress (6 per tet) for tets with |det J_ref| >= 1e-30; others are left
 * as they are.  J of the stress is det F_sl3 (the reference passes an
 * uninitialized value).  Returns the count of |det F_sl3 - 1| > 1e-8. */
uint32_t orc_element_states(uint32_t n_nodes, uint32_t n_elems, const double* xyz,
                            const uint32_t* conn, const double* mu_e, const double* lam_e,
                            const double* u, double* Fst, double* stress) {
    (void)n_nodes;
    static const double xi[4][3] = {{-1, -1, -1}, {1, 0, 0}, {0, 1, 0}, {0, 0, 1}};
    uint32_t bad = 0;
    for (uint32_t e = 0; e < n_elems; ++e) {
        const uint32_t* c = conn + 4 * (size_t)e;
        double x[4][3], ue[4][3], J[9], Ji[9], dN[4][3], g[9];
        for (int a = 0; a < 4; ++a)
            for (int d = 0; d < 3; ++d) {
                x[a][d] = xyz[3 * (size_t)c[a] + d];
                ue[a][d] = u[3 * (size_t)c[a] + d];
            }
        for (int d = 0; d < 3; ++d) {
            J[d * 3 + 0] = x[1][d] - x[0][d];
            J[d * 3 + 1] = x[2][d] - x[0][d];
            J[d * 3 + 2] = x[3][d] - x[0][d];
        }
        orc_inv3(J, Ji);
        const double dJ = J[0] * (J[4] * J[8] - J[7] * J[5]) - J[3] * (J[1] * J[8] - J[7] * J[2]) +
                          J[6] * (J[1] * J[5] - J[4] * J[2]);
        if (fabs(dJ) < 1e-30) continue;
        for (int a = 0; a < 4; ++a)
            for (int i = 0; i < 3; ++i) {
                double s = 0.0;
                for (int j = 0; j < 3; ++j) s += Ji[j * 3 + i] * xi[a][j];
                dN[a][i] = s;
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double s = 0.0;
                for (int a = 0; a < 4; ++a) s += ue[a][i] * dN[a][j];
                g[i * 3 + j] = s;
            }
        double F[9], Fs[9];
        for (int i = 0; i < 9; ++i) F[i] = (i % 4 == 0) ? 1.0 + g[i] : g[i];
        orc_sl3_retraction(F, Fs);
        orc_m3 fs;
        memcpy(fs.a, Fs, sizeof fs.a);
        const double dF = m3_det(fs);
        orc_nh_response(Fs, mu_e[e], lam_e[e], dF, stress + 6 * (size_t)e);
        memcpy(Fst + 9 * (size_t)e, Fs, sizeof Fs);
        if (fabs(dF - 1.0) > 1.0e-8) ++bad;
    }
    return bad;
}
