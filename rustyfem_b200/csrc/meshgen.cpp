// Synthetic FEM workloads for the multifrontal solver: structured meshes of
// linear-elastic solids, assembled into the lower-triangle CSC that the
// RustyFEM C interface takes (caller numbering, one column per free DOF), plus
// the engine-side node graph (coordinates, neighbour lists, DOFs per node).
//
// The element formulations follow the reference:
//  * C3D8: trilinear hexahedron, 2×2×2 Gauss points with volumetric B-bar
//    (src/elements/continuum3d.rs:39-84, 116-120; src/elements/common.rs:142-200, 252-289),
//  * C3D20: 20-node serendipity hexahedron, 3×3×3 Gauss points
//    (src/elements/solid_higher.rs:113, 137-183; solid_higher_shapes.rs:190-205, 279-287),
//  * CPS4: bilinear quadrilateral in plane stress, 2×2 Gauss points, weight det·t
//    (src/elements/continuum2d.rs:25, 34-60),
//  * isotropic elasticity (src/materials/elastic.rs:47-72),
//  * meshes as `box_solid` (src/model.rs:454-500, nodes x fastest) and `plate`
//    (src/model.rs:397-451, rows of nodes along x),
//  * free DOFs numbered node by node (src/fem/assembly.rs:245-253): nodes on
//    the plane x = 0 are clamped and carry no DOF,
//  * a total force spread over a face as uniform pressure (src/model.rs:811-858):
//    nodal weights are the integrals of the face shape functions.
// Every element of a structured mesh has the same geometry, so the unit
// stiffness (E = 1) is integrated once and scaled per element by its E.

#include <algorithm>
#include <array>
#include <cmath>
#include <cstdint>
#include <cstring>
#include <vector>

namespace {

using std::size_t;
using std::vector;

const double G2 = 0.5773502691896258;  // 1/sqrt(3)

struct Mesh {
    int dim = 3;  // displacement components per node
    vector<double> xyz;               // 3 per node
    vector<vector<size_t>> elems;     // node lists
    vector<double> emod;              // Young's modulus per element
    vector<uint8_t> clamped;          // per node
    vector<double> ke_unit;           // stiffness of one element for E = 1 (nd × nd, row-major)
    size_t nen = 0;                   // nodes per element
    vector<double> fnode;             // dim per node: applied nodal force
    // assembled
    vector<int64_t> dof_first;        // per node: first free DOF or -1
    size_t n = 0;
    vector<int64_t> loc;              // dof -> node
    vector<int64_t> indptr, indices;
    vector<double> data;
    vector<double> rhs;
    // graph form
    vector<int64_t> blocks;           // free nodes
    vector<int64_t> adj_ptr, adj_idx;
};

void inv3(const double m[3][3], double inv[3][3], double* det) {
    double d = m[0][0] * (m[1][1] * m[2][2] - m[1][2] * m[2][1]) - m[0][1] * (m[1][0] * m[2][2] - m[1][2] * m[2][0]) +
               m[0][2] * (m[1][0] * m[2][1] - m[1][1] * m[2][0]);
    double id = 1.0 / d;
    inv[0][0] = (m[1][1] * m[2][2] - m[1][2] * m[2][1]) * id;
    inv[0][1] = (m[0][2] * m[2][1] - m[0][1] * m[2][2]) * id;
    inv[0][2] = (m[0][1] * m[1][2] - m[0][2] * m[1][1]) * id;
    inv[1][0] = (m[1][2] * m[2][0] - m[1][0] * m[2][2]) * id;
    inv[1][1] = (m[0][0] * m[2][2] - m[0][2] * m[2][0]) * id;
    inv[1][2] = (m[0][2] * m[1][0] - m[0][0] * m[1][2]) * id;
    inv[2][0] = (m[1][0] * m[2][1] - m[1][1] * m[2][0]) * id;
    inv[2][1] = (m[0][1] * m[2][0] - m[0][0] * m[2][1]) * id;
    inv[2][2] = (m[0][0] * m[1][1] - m[0][1] * m[1][0]) * id;
    *det = d;
}

// isotropic 3D elasticity, components xx yy zz xy xz yz
void dmat3(double E, double nu, double D[6][6]) {
    double lam = E * nu / ((1.0 + nu) * (1.0 - 2.0 * nu));
    double mu = E / (2.0 * (1.0 + nu));
    memset(D, 0, sizeof(double) * 36);
    for (int i = 0; i < 3; i++) {
        for (int j = 0; j < 3; j++) D[i][j] = lam;
        D[i][i] = lam + 2.0 * mu;
    }
    for (int i = 3; i < 6; i++) D[i][i] = mu;
}

// Ke += w Bᵀ D B  (B ns × nd row-major)
void add_btdb(vector<double>& ke, const vector<double>& B, const double* D, int ns, int nd, double w) {
    vector<double> db(ns * nd, 0.0);
    for (int r = 0; r < ns; r++)
        for (int m = 0; m < ns; m++) {
            double drm = D[r * ns + m];
            if (drm != 0.0)
                for (int c = 0; c < nd; c++) db[r * nd + c] += drm * B[m * nd + c];
        }
    for (int r = 0; r < ns; r++)
        for (int i = 0; i < nd; i++) {
            double bri = B[r * nd + i] * w;
            if (bri != 0.0)
                for (int j = 0; j < nd; j++) ke[i * nd + j] += bri * db[r * nd + j];
        }
}

// 3D B matrix (6 × 3nn) from dN/dx
vector<double> bmat3(const vector<std::array<double, 3>>& dndx) {
    int nn = (int)dndx.size(), nd = 3 * nn;
    vector<double> b(6 * nd, 0.0);
    for (int i = 0; i < nn; i++) {
        const auto& d = dndx[i];
        int c = 3 * i;
        b[c] = d[0];
        b[nd + c + 1] = d[1];
        b[2 * nd + c + 2] = d[2];
        b[3 * nd + c] = d[1];
        b[3 * nd + c + 1] = d[0];
        b[4 * nd + c] = d[2];
        b[4 * nd + c + 2] = d[0];
        b[5 * nd + c + 1] = d[2];
        b[5 * nd + c + 2] = d[1];
    }
    return b;
}

const double HEX_C[8][3] = {{-1, -1, -1}, {1, -1, -1}, {1, 1, -1}, {-1, 1, -1},
                            {-1, -1, 1},  {1, -1, 1},  {1, 1, 1},  {-1, 1, 1}};
const double HEX20_MID[12][3] = {{0, -1, -1}, {1, 0, -1}, {0, 1, -1}, {-1, 0, -1}, {0, -1, 1}, {1, 0, 1},
                                 {0, 1, 1},   {-1, 0, 1}, {-1, -1, 0}, {1, -1, 0}, {1, 1, 0}, {-1, 1, 0}};

struct Ip {
    vector<std::array<double, 3>> dndx;
    double w;
};

// isoparametric 3D point: dn[i][r] = dN_i/dξ_r
Ip ip3(const vector<std::array<double, 3>>& x, const vector<std::array<double, 3>>& dn, double gw) {
    size_t nn = x.size();
    double J[3][3] = {};
    for (int r = 0; r < 3; r++)
        for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (size_t i = 0; i < nn; i++) s += dn[i][r] * x[i][c];
            J[r][c] = s;
        }
    double ji[3][3], det;
    inv3(J, ji, &det);
    Ip ip;
    ip.dndx.resize(nn);
    for (size_t i = 0; i < nn; i++)
        for (int c = 0; c < 3; c++) {
            double s = 0.0;
            for (int r = 0; r < 3; r++) s += ji[c][r] * dn[i][r];
            ip.dndx[i][c] = s;
        }
    ip.w = det * gw;
    return ip;
}

// C3D8 with volumetric B-bar, E = 1
vector<double> ke_hex8(const vector<std::array<double, 3>>& x, double nu) {
    vector<Ip> ips;
    const double gp[2] = {-G2, G2};
    for (double zeta : gp)
        for (double eta : gp)
            for (double xi : gp) {
                vector<std::array<double, 3>> dn(8);
                double p[3] = {xi, eta, zeta};
                for (int i = 0; i < 8; i++) {
                    const double* nat = HEX_C[i];
                    double f0 = 1.0 + p[0] * nat[0], f1 = 1.0 + p[1] * nat[1], f2 = 1.0 + p[2] * nat[2];
                    dn[i] = {0.125 * nat[0] * f1 * f2, 0.125 * nat[1] * f0 * f2, 0.125 * nat[2] * f0 * f1};
                }
                ips.push_back(ip3(x, dn, 1.0));
            }
    int nd = 24;
    vector<vector<double>> bs;
    for (auto& ip : ips) bs.push_back(bmat3(ip.dndx));
    // volumetric B-bar (src/elements/common.rs:177-200)
    auto vol = [&](const vector<double>& b, int c) { return b[c] + b[nd + c] + b[2 * nd + c]; };
    double wsum = 0.0;
    for (auto& ip : ips) wsum += ip.w;
    vector<double> avg(nd);
    for (int c = 0; c < nd; c++) {
        double s = 0.0;
        for (size_t q = 0; q < ips.size(); q++) s += ips[q].w * vol(bs[q], c);
        avg[c] = s / wsum;
    }
    for (auto& b : bs)
        for (int c = 0; c < nd; c++) {
            double corr = (avg[c] - vol(b, c)) / 3.0;
            for (int r = 0; r < 3; r++) b[r * nd + c] += corr;
        }
    double D[6][6];
    dmat3(1.0, nu, D);
    vector<double> ke(nd * nd, 0.0);
    for (size_t q = 0; q < ips.size(); q++) add_btdb(ke, bs[q], &D[0][0], 6, nd, ips[q].w);
    return ke;
}

// C3D20, 3×3×3 Gauss, E = 1
vector<double> ke_hex20(const vector<std::array<double, 3>>& x, double nu) {
    const double g = std::sqrt(0.6);
    const double gx[3] = {-g, 0.0, g}, gw[3] = {5.0 / 9.0, 8.0 / 9.0, 5.0 / 9.0};
    double D[6][6];
    dmat3(1.0, nu, D);
    int nd = 60;
    vector<double> ke(nd * nd, 0.0);
    for (int a = 0; a < 3; a++)
        for (int b2 = 0; b2 < 3; b2++)
            for (int c = 0; c < 3; c++) {
                double p[3] = {gx[c], gx[b2], gx[a]};
                double w = gw[a] * gw[b2] * gw[c];
                vector<std::array<double, 3>> dn(20);
                for (int i = 0; i < 8; i++) {
                    const double* h = HEX_C[i];
                    double f[3] = {1.0 + p[0] * h[0], 1.0 + p[1] * h[1], 1.0 + p[2] * h[2]};
                    double s = p[0] * h[0] + p[1] * h[1] + p[2] * h[2] - 2.0;
                    for (int r = 0; r < 3; r++) {
                        // d/dp_r [f0 f1 f2 s]/8
                        double prod_other = 1.0;
                        for (int q = 0; q < 3; q++)
                            if (q != r) prod_other *= f[q];
                        dn[i][r] = 0.125 * (h[r] * prod_other * s + f[0] * f[1] * f[2] * h[r]);
                    }
                }
                for (int mi = 0; mi < 12; mi++) {
                    const double* m = HEX20_MID[mi];
                    double fq[3], dfq[3];
                    for (int q = 0; q < 3; q++) {
                        if (m[q] == 0.0) {
                            fq[q] = 1.0 - p[q] * p[q];
                            dfq[q] = -2.0 * p[q];
                        } else {
                            fq[q] = 1.0 + p[q] * m[q];
                            dfq[q] = m[q];
                        }
                    }
                    dn[8 + mi] = {0.25 * dfq[0] * fq[1] * fq[2], 0.25 * fq[0] * dfq[1] * fq[2], 0.25 * fq[0] * fq[1] * dfq[2]};
                }
                Ip ip = ip3(x, dn, w);
                add_btdb(ke, bmat3(ip.dndx), &D[0][0], 6, nd, ip.w);
            }
    return ke;
}

// CPS4 plane stress, thickness t, E = 1
vector<double> ke_cps4(const vector<std::array<double, 3>>& x, double nu, double t) {
    const double nat[4][2] = {{-1, -1}, {1, -1}, {1, 1}, {-1, 1}};
    const double pts[4][2] = {{-G2, -G2}, {G2, -G2}, {-G2, G2}, {G2, G2}};
    double c = 1.0 / (1.0 - nu * nu);
    double D[9] = {c, c * nu, 0.0, c * nu, c, 0.0, 0.0, 0.0, c * (1.0 - nu) / 2.0};
    int nd = 8;
    vector<double> ke(nd * nd, 0.0);
    for (auto& pt : pts) {
        double xi = pt[0], eta = pt[1];
        double dxi[4], deta[4];
        for (int i = 0; i < 4; i++) {
            dxi[i] = 0.25 * nat[i][0] * (1.0 + eta * nat[i][1]);
            deta[i] = 0.25 * nat[i][1] * (1.0 + xi * nat[i][0]);
        }
        double j[2][2] = {};
        for (int i = 0; i < 4; i++) {
            j[0][0] += dxi[i] * x[i][0];
            j[0][1] += dxi[i] * x[i][1];
            j[1][0] += deta[i] * x[i][0];
            j[1][1] += deta[i] * x[i][1];
        }
        double det = j[0][0] * j[1][1] - j[0][1] * j[1][0];
        vector<double> B(3 * nd, 0.0);
        for (int i = 0; i < 4; i++) {
            double d0 = (j[1][1] * dxi[i] - j[0][1] * deta[i]) / det;
            double d1 = (-j[1][0] * dxi[i] + j[0][0] * deta[i]) / det;
            B[2 * i] = d0;
            B[nd + 2 * i + 1] = d1;
            B[2 * nd + 2 * i] = d1;
            B[2 * nd + 2 * i + 1] = d0;
        }
        add_btdb(ke, B, D, 3, nd, det * t);
    }
    return ke;
}

// Numbering, CSC lower (caller numbering), graph and RHS.
void assemble(Mesh& M) {
    size_t nn = M.xyz.size() / 3;
    int dim = M.dim;
    M.dof_first.assign(nn, -1);
    size_t n = 0;
    for (size_t v = 0; v < nn; v++)
        if (!M.clamped[v]) {
            M.dof_first[v] = (int64_t)n;
            n += dim;
            M.blocks.push_back((int64_t)v);
        }
    M.n = n;
    M.loc.resize(n);
    for (size_t v = 0; v < nn; v++)
        if (M.dof_first[v] >= 0)
            for (int s = 0; s < dim; s++) M.loc[M.dof_first[v] + s] = (int64_t)v;
    // neighbour lists (both directions, excluding the node itself) of free nodes
    vector<vector<size_t>> nb(nn);
    for (auto& e : M.elems)
        for (size_t a : e) {
            if (M.clamped[a]) continue;
            for (size_t b : e)
                if (b != a && !M.clamped[b]) nb[a].push_back(b);
        }
    for (auto& l : nb) {
        std::sort(l.begin(), l.end());
        l.erase(std::unique(l.begin(), l.end()), l.end());
    }
    // graph form: block ids are positions among free nodes
    vector<int64_t> bid(nn, -1);
    for (size_t i = 0; i < M.blocks.size(); i++) bid[M.blocks[i]] = (int64_t)i;
    M.adj_ptr.assign(M.blocks.size() + 1, 0);
    for (size_t i = 0; i < M.blocks.size(); i++) {
        for (size_t w : nb[M.blocks[i]]) M.adj_idx.push_back(bid[w]);
        M.adj_ptr[i + 1] = (int64_t)M.adj_idx.size();
    }
    // upper node neighbours (w >= v, v itself first) with dim×dim blocks
    vector<vector<size_t>> up(nn);
    vector<size_t> boff(nn + 1, 0);
    for (size_t v = 0; v < nn; v++) {
        if (M.clamped[v]) continue;
        up[v].push_back(v);
        for (size_t w : nb[v])
            if (w > v) up[v].push_back(w);
    }
    for (size_t v = 0; v < nn; v++) boff[v + 1] = boff[v] + up[v].size();
    vector<double> blk(boff[nn] * dim * dim, 0.0);  // block (v, w): [sw][sv] = K(dof(w,sw), dof(v,sv))
    size_t nen = M.nen, nd = nen * dim;
    for (size_t ei = 0; ei < M.elems.size(); ei++) {
        const auto& e = M.elems[ei];
        double E = M.emod[ei];
        for (size_t a = 0; a < nen; a++) {
            size_t va = e[a];
            if (M.clamped[va]) continue;
            for (size_t b = 0; b < nen; b++) {
                size_t vb = e[b];
                if (M.clamped[vb] || vb < va) continue;
                auto it = std::lower_bound(up[va].begin() + 1, up[va].end(), vb);
                size_t idx = (vb == va) ? 0 : (size_t)(it - up[va].begin());
                double* B = blk.data() + (boff[va] + idx) * dim * dim;
                for (int sb = 0; sb < dim; sb++)
                    for (int sa = 0; sa < dim; sa++) B[sb * dim + sa] += E * M.ke_unit[(b * dim + sb) * nd + a * dim + sa];
            }
        }
    }
    M.indptr.assign(n + 1, 0);
    for (size_t v = 0; v < nn; v++) {
        if (M.clamped[v]) continue;
        for (int sa = 0; sa < dim; sa++) {
            size_t c = (size_t)M.dof_first[v] + sa;
            for (size_t idx = 0; idx < up[v].size(); idx++) {
                size_t w = up[v][idx];
                const double* B = blk.data() + (boff[v] + idx) * dim * dim;
                for (int sb = 0; sb < dim; sb++) {
                    size_t r = (size_t)M.dof_first[w] + sb;
                    if (r < c) continue;
                    M.indices.push_back((int64_t)r);
                    M.data.push_back(B[sb * dim + sa]);
                }
            }
            M.indptr[c + 1] = (int64_t)M.indices.size();
        }
    }
    M.rhs.assign(n, 0.0);
    for (size_t v = 0; v < nn; v++)
        if (M.dof_first[v] >= 0)
            for (int s = 0; s < dim; s++) M.rhs[M.dof_first[v] + s] = M.fnode[v * dim + s];
}

}  // namespace

extern "C" {

// n×n×n C3D8 on the unit cube (n+1)³ nodes; x = 0 clamped; total force fz
// spread over the face x = 1. `emod` (n³, element order i fastest) may be
// null for a homogeneous E.
void* rfg_mesh_hex8_cube(int64_t n, double E, double nu, const double* emod, double fz) {
    Mesh* M = new Mesh();
    M->dim = 3;
    M->nen = 8;
    size_t np = (size_t)n + 1;
    auto id = [&](size_t i, size_t j, size_t k) { return (k * np + j) * np + i; };
    M->xyz.resize(3 * np * np * np);
    M->clamped.assign(np * np * np, 0);
    for (size_t k = 0; k < np; k++)
        for (size_t j = 0; j < np; j++)
            for (size_t i = 0; i < np; i++) {
                size_t v = id(i, j, k);
                M->xyz[3 * v] = (double)i / (double)n;
                M->xyz[3 * v + 1] = (double)j / (double)n;
                M->xyz[3 * v + 2] = (double)k / (double)n;
                M->clamped[v] = (i == 0);
            }
    size_t ne = (size_t)n * n * n;
    M->elems.reserve(ne);
    for (size_t k = 0; k < (size_t)n; k++)
        for (size_t j = 0; j < (size_t)n; j++)
            for (size_t i = 0; i < (size_t)n; i++)
                M->elems.push_back({id(i, j, k), id(i + 1, j, k), id(i + 1, j + 1, k), id(i, j + 1, k), id(i, j, k + 1),
                                    id(i + 1, j, k + 1), id(i + 1, j + 1, k + 1), id(i, j + 1, k + 1)});
    M->emod.resize(ne);
    for (size_t e = 0; e < ne; e++) M->emod[e] = emod ? emod[e] : E;
    vector<std::array<double, 3>> x(8);
    for (int a = 0; a < 8; a++)
        for (int c = 0; c < 3; c++) x[a][c] = M->xyz[3 * M->elems[0][a] + c];
    M->ke_unit = ke_hex8(x, nu);
    // uniform pressure on x = 1: bilinear face weights h²/4 per facet corner
    M->fnode.assign(3 * np * np * np, 0.0);
    vector<double> w(np * np * np, 0.0);
    double total = 0.0;
    for (size_t k = 0; k < (size_t)n; k++)
        for (size_t j = 0; j < (size_t)n; j++) {
            size_t f[4] = {id(n, j, k), id(n, j + 1, k), id(n, j + 1, k + 1), id(n, j, k + 1)};
            double a = 1.0 / ((double)n * n) / 4.0;
            for (size_t v : f) {
                w[v] += a;
                total += a;
            }
        }
    for (size_t v = 0; v < w.size(); v++)
        if (w[v] != 0.0) M->fnode[3 * v + 2] = fz * w[v] / total;
    assemble(*M);
    return M;
}

// n×n×n C3D20 (serendipity) on the unit cube; x = 0 clamped; total force fz
// spread over the face x = 1 with the 8-node face's consistent weights.
void* rfg_mesh_hex20_cube(int64_t n, double E, double nu, double fz) {
    Mesh* M = new Mesh();
    M->dim = 3;
    M->nen = 20;
    size_t L = 2 * (size_t)n + 1;  // lattice points per axis
    vector<int64_t> lid(L * L * L, -1);
    auto lat = [&](size_t i, size_t j, size_t k) { return (k * L + j) * L + i; };
    size_t nn = 0;
    for (size_t k = 0; k < L; k++)
        for (size_t j = 0; j < L; j++)
            for (size_t i = 0; i < L; i++) {
                int odd = (int)(i & 1) + (int)(j & 1) + (int)(k & 1);
                if (odd > 1) continue;
                lid[lat(i, j, k)] = (int64_t)nn++;
                M->xyz.push_back((double)i / (double)(2 * n));
                M->xyz.push_back((double)j / (double)(2 * n));
                M->xyz.push_back((double)k / (double)(2 * n));
                M->clamped.push_back(i == 0);
            }
    for (size_t k = 0; k < (size_t)n; k++)
        for (size_t j = 0; j < (size_t)n; j++)
            for (size_t i = 0; i < (size_t)n; i++) {
                vector<size_t> e;
                for (int a = 0; a < 8; a++)
                    e.push_back((size_t)lid[lat(2 * i + (HEX_C[a][0] > 0 ? 2 : 0), 2 * j + (HEX_C[a][1] > 0 ? 2 : 0),
                                                2 * k + (HEX_C[a][2] > 0 ? 2 : 0))]);
                for (int a = 0; a < 12; a++)
                    e.push_back((size_t)lid[lat(2 * i + 1 + (int)HEX20_MID[a][0], 2 * j + 1 + (int)HEX20_MID[a][1],
                                                2 * k + 1 + (int)HEX20_MID[a][2])]);
                M->elems.push_back(e);
            }
    M->emod.assign(M->elems.size(), E);
    vector<std::array<double, 3>> x(20);
    for (int a = 0; a < 20; a++)
        for (int c = 0; c < 3; c++) x[a][c] = M->xyz[3 * M->elems[0][a] + c];
    M->ke_unit = ke_hex20(x, nu);
    // consistent weights of an 8-node quad face: corners -A/12, midsides A/3
    M->fnode.assign(3 * nn, 0.0);
    vector<double> w(nn, 0.0);
    double A = 1.0 / ((double)n * n), total = 0.0;
    for (size_t k = 0; k < (size_t)n; k++)
        for (size_t j = 0; j < (size_t)n; j++) {
            size_t i = L - 1;
            size_t corners[4] = {lat(i, 2 * j, 2 * k), lat(i, 2 * j + 2, 2 * k), lat(i, 2 * j + 2, 2 * k + 2), lat(i, 2 * j, 2 * k + 2)};
            size_t mids[4] = {lat(i, 2 * j + 1, 2 * k), lat(i, 2 * j + 2, 2 * k + 1), lat(i, 2 * j + 1, 2 * k + 2), lat(i, 2 * j, 2 * k + 1)};
            for (size_t c : corners) {
                w[lid[c]] += -A / 12.0;
                total += -A / 12.0;
            }
            for (size_t c : mids) {
                w[lid[c]] += A / 3.0;
                total += A / 3.0;
            }
        }
    for (size_t v = 0; v < nn; v++)
        if (w[v] != 0.0) M->fnode[3 * v + 2] = fz * w[v] / total;
    assemble(*M);
    return M;
}

// nx×ny CPS4 plate of element size h and thickness t in the x–y plane;
// x = 0 edge clamped; total force fy spread over the edge x = nx·h.
void* rfg_mesh_plate(int64_t nx, int64_t ny, double h, double t, double E, double nu, double fy) {
    Mesh* M = new Mesh();
    M->dim = 2;
    M->nen = 4;
    size_t px = (size_t)nx + 1, py = (size_t)ny + 1;
    auto id = [&](size_t i, size_t j) { return j * px + i; };
    double Lx = (double)nx * h, Ly = (double)ny * h;
    for (size_t j = 0; j < py; j++)
        for (size_t i = 0; i < px; i++) {
            double s = (double)i / (double)nx, tt = (double)j / (double)ny;
            M->xyz.push_back(s * Lx);
            M->xyz.push_back(tt * Ly);
            M->xyz.push_back(0.0);
            M->clamped.push_back(i == 0);
        }
    for (size_t j = 0; j < (size_t)ny; j++)
        for (size_t i = 0; i < (size_t)nx; i++) M->elems.push_back({id(i, j), id(i + 1, j), id(i + 1, j + 1), id(i, j + 1)});
    M->emod.assign(M->elems.size(), E);
    vector<std::array<double, 3>> x(4);
    for (int a = 0; a < 4; a++)
        for (int c = 0; c < 3; c++) x[a][c] = M->xyz[3 * M->elems[0][a] + c];
    M->ke_unit = ke_cps4(x, nu, t);
    size_t nn = px * py;
    M->fnode.assign(2 * nn, 0.0);
    vector<double> w(nn, 0.0);
    double total = 0.0;
    for (size_t j = 0; j < (size_t)ny; j++) {
        double a = Ly / (double)ny / 2.0;
        w[id(nx, j)] += a;
        w[id(nx, j + 1)] += a;
        total += 2.0 * a;
    }
    for (size_t v = 0; v < nn; v++)
        if (w[v] != 0.0) M->fnode[2 * v + 1] = fy * w[v] / total;
    assemble(*M);
    return M;
}

size_t rfg_mesh_n(const void* h) { return ((const Mesh*)h)->n; }
size_t rfg_mesh_nn(const void* h) { return ((const Mesh*)h)->xyz.size() / 3; }
size_t rfg_mesh_nnz(const void* h) { return ((const Mesh*)h)->indices.size(); }
size_t rfg_mesh_nelem(const void* h) { return ((const Mesh*)h)->elems.size(); }
size_t rfg_mesh_nblocks(const void* h) { return ((const Mesh*)h)->blocks.size(); }
size_t rfg_mesh_adj_nnz(const void* h) { return ((const Mesh*)h)->adj_idx.size(); }
int64_t rfg_mesh_dim(const void* h) { return ((const Mesh*)h)->dim; }

// The C-interface form: loc[n], coords[3nn], CSC lower indptr[n+1], indices/data[nnz], rhs[n].
void rfg_mesh_export(const void* hp, int64_t* loc, double* coords, int64_t* indptr, int64_t* indices, double* data,
                     double* rhs) {
    const Mesh* M = (const Mesh*)hp;
    if (loc) std::copy(M->loc.begin(), M->loc.end(), loc);
    if (coords) std::copy(M->xyz.begin(), M->xyz.end(), coords);
    if (indptr) std::copy(M->indptr.begin(), M->indptr.end(), indptr);
    if (indices) std::copy(M->indices.begin(), M->indices.end(), indices);
    if (data) std::copy(M->data.begin(), M->data.end(), data);
    if (rhs) std::copy(M->rhs.begin(), M->rhs.end(), rhs);
}

// The engine form: per free node (block) its coordinates, sorted neighbours and DOF count.
void rfg_mesh_graph(const void* hp, double* coords, int64_t* adj_ptr, int64_t* adj_idx, int64_t* ndof) {
    const Mesh* M = (const Mesh*)hp;
    for (size_t i = 0; i < M->blocks.size(); i++) {
        size_t v = (size_t)M->blocks[i];
        for (int c = 0; c < 3; c++) coords[3 * i + c] = M->xyz[3 * v + c];
        ndof[i] = M->dim;
    }
    std::copy(M->adj_ptr.begin(), M->adj_ptr.end(), adj_ptr);
    std::copy(M->adj_idx.begin(), M->adj_idx.end(), adj_idx);
}

void rfg_mesh_free(void* h) { delete (Mesh*)h; }

}  // extern "C"
