// Test-matrix generators and the reference's binary system format.
//
// gen_cube restates examples/common/generator/cube.inl:69-230: cell-centred
// finite-volume 7-point diffusion on an nx*ny*nz grid, row order "diagonal
// first, then b, s, w, e, n, t" (ascending column after the diagonal),
// Dirichlet faces folded into the diagonal as 2*q*K, q = a/h^2.
// gen_7pt_faces uses the same assembly with caller-supplied face
// coefficients (variable-coefficient and bump-field problems).
// gen_27pt builds the 27-point anisotropic operator of the 128^3 benchmark,
// which has no counterpart in the reference (see the function comment).
#include "common.h"
#include <cmath>

namespace xamg {

static double cube_K(double xc, double yc, double zc, int mode) {
    double val = 1.0;
    if (mode == 3) {
        if (xc >= 0.1 && xc <= 0.9 && yc >= 0.1 && yc <= 0.9 && zc >= 0.1 && zc <= 0.9)
            val = 1e3;
        else {
            bool cx = xc < 0.1 || xc > 0.9, cy = yc < 0.1 || yc > 0.9, cz = zc < 0.1 || zc > 0.9;
            if (cx && cy && cz) val = 1e-2;
        }
    } else if (mode == 4) {
        if (xc >= 1. / 3. && xc <= 2. / 3. && yc >= 1. / 3. && yc <= 2. / 3. && zc >= 1. / 3. &&
            zc <= 2. / 3.)
            val = 1e-8;
    }
    return val;
}

// Face coefficient callback: face of cell (i,j,k) in direction dir (0=b,1=s,
// 2=w,3=e,4=n,5=t).
template <class FK>
static void assemble_7pt(i64 nx, i64 ny, i64 nz, double q1, double q2, double q3, FK K,
                         HostCsr &A) {
    i64 n = nx * ny * nz;
    A.n = A.ncols = n;
    A.rp.assign(n + 1, 0);
    for (i64 r = 0; r < n; ++r) {
        i64 ii = r % nx, jj = (r / nx) % ny, kk = r / (nx * ny);
        int c = 1 + (kk > 0) + (jj > 0) + (ii > 0) + (ii < nx - 1) + (jj < ny - 1) + (kk < nz - 1);
        A.rp[r + 1] = A.rp[r] + c;
    }
    A.ci.resize(A.rp[n]);
    A.v.resize(A.rp[n]);
    for (i64 r = 0; r < n; ++r) {
        i64 ii = r % nx, jj = (r / nx) % ny, kk = r / (nx * ny);
        int p = A.rp[r];
        int d = p++;
        A.ci[d] = (int)r;
        double diag = 0.0;
        auto link = [&](bool inside, double q, double k, i64 col) {
            if (inside) {
                diag += q * k;
                A.ci[p] = (int)col;
                A.v[p] = -q * k;
                ++p;
            }
        };
        double Kb = K(ii, jj, kk, 0), Ks = K(ii, jj, kk, 1), Kw = K(ii, jj, kk, 2),
               Ke = K(ii, jj, kk, 3), Kn = K(ii, jj, kk, 4), Kt = K(ii, jj, kk, 5);
        if (kk > 0) link(true, q3, Kb, r - nx * ny); else if (nz > 1) diag += 2.0 * q3 * Kb;
        if (jj > 0) link(true, q2, Ks, r - nx); else if (ny > 1) diag += 2.0 * q2 * Ks;
        if (ii > 0) link(true, q1, Kw, r - 1); else if (nx > 1) diag += 2.0 * q1 * Kw;
        if (ii < nx - 1) link(true, q1, Ke, r + 1); else if (nx > 1) diag += 2.0 * q1 * Ke;
        if (jj < ny - 1) link(true, q2, Kn, r + nx); else if (ny > 1) diag += 2.0 * q2 * Kn;
        if (kk < nz - 1) link(true, q3, Kt, r + nx * ny); else if (nz > 1) diag += 2.0 * q3 * Kt;
        A.v[d] = diag;
    }
}

void gen_cube(i64 nx, i64 ny, i64 nz, int config, HostCsr &A) {
    double aa[3] = {1.0, 1.0, 1.0};
    if (config == 1) { aa[0] = 0.1; aa[2] = 10; }
    else if (config == 2) aa[0] = 1e-3;
    double hx = 1.0 / nx, hy = 1.0 / ny, hz = 1.0 / nz;
    double q1 = aa[0] / hx / hx, q2 = aa[1] / hy / hy, q3 = aa[2] / hz / hz;
    auto K = [&](i64 i, i64 j, i64 k, int dir) {
        double xc = hx * (i + 0.5), yc = hy * (j + 0.5), zc = hz * (k + 0.5);
        switch (dir) {
        case 0: zc -= 0.5 * hz; break;
        case 1: yc -= 0.5 * hy; break;
        case 2: xc -= 0.5 * hx; break;
        case 3: xc += 0.5 * hx; break;
        case 4: yc += 0.5 * hy; break;
        default: zc += 0.5 * hz; break;
        }
        return cube_K(xc, yc, zc, config);
    };
    assemble_7pt(nx, ny, nz, q1, q2, q3, K, A);
}

// Face coefficients: kx[(k*ny + j)*(nx+1) + i] is the face between cells i-1
// and i of row (j,k) (i = 0 and i = nx are the domain faces); ky, kz alike.
void gen_7pt_faces(i64 nx, i64 ny, i64 nz, const double *kx, const double *ky, const double *kz,
                   HostCsr &A) {
    double q1 = (double)nx * nx, q2 = (double)ny * ny, q3 = (double)nz * nz;
    auto K = [&](i64 i, i64 j, i64 k, int dir) {
        switch (dir) {
        case 0: return kz[(k * ny + j) * nx + i];            // z face k
        case 1: return ky[(k * (ny + 1) + j) * nx + i];      // y face j
        case 2: return kx[(k * ny + j) * (nx + 1) + i];      // x face i
        case 3: return kx[(k * ny + j) * (nx + 1) + i + 1];  // x face i+1
        case 4: return ky[(k * (ny + 1) + j + 1) * nx + i];  // y face j+1
        default: return kz[((k + 1) * ny + j) * nx + i];     // z face k+1
        }
    };
    assemble_7pt(nx, ny, nz, q1, q2, q3, K, A);
}

// 27-point anisotropic diffusion on an n^3 grid with Dirichlet boundary.
// Neighbour offset d = (dx,dy,dz) in {-1,0,1}^3 \ 0 couples with weight
//   w_d = (kx*dx^2 + ky*dy^2 + kz*dz^2) / |d|^4,
// i.e. the sum over the 13 lattice directions of a K-projected second
// difference; a_ij = -w_d and the diagonal is the sum of w_d over all 26
// offsets (neighbours outside the box are eliminated, keeping their weight on
// the diagonal).  The result is a symmetric M-matrix.  Row order: diagonal
// first, then the remaining columns ascending.
void gen_27pt(i64 n, double kx, double ky, double kz, HostCsr &A) {
    i64 N = n * n * n;
    A.n = A.ncols = N;
    A.rp.assign(N + 1, 0);
    double w[27];
    double dsum = 0.0;
    for (int dz = -1; dz <= 1; ++dz)
        for (int dy = -1; dy <= 1; ++dy)
            for (int dx = -1; dx <= 1; ++dx) {
                int q = (dz + 1) * 9 + (dy + 1) * 3 + (dx + 1);
                int d2 = dx * dx + dy * dy + dz * dz;
                w[q] = d2 ? (kx * dx * dx + ky * dy * dy + kz * dz * dz) / double(d2 * d2) : 0.0;
                dsum += w[q];
            }
    for (i64 r = 0; r < N; ++r) {
        i64 i = r % n, j = (r / n) % n, k = r / (n * n);
        int cx = 1 + (i > 0) + (i < n - 1), cy = 1 + (j > 0) + (j < n - 1), cz = 1 + (k > 0) + (k < n - 1);
        A.rp[r + 1] = A.rp[r] + cx * cy * cz;
    }
    A.ci.resize(A.rp[N]);
    A.v.resize(A.rp[N]);
    for (i64 r = 0; r < N; ++r) {
        i64 i = r % n, j = (r / n) % n, k = r / (n * n);
        int p = A.rp[r];
        A.ci[p] = (int)r;
        A.v[p] = dsum;
        ++p;
        for (int dz = -1; dz <= 1; ++dz)
            for (int dy = -1; dy <= 1; ++dy)
                for (int dx = -1; dx <= 1; ++dx) {
                    if (!dx && !dy && !dz) continue;
                    i64 ii = i + dx, jj = j + dy, kk = k + dz;
                    if (ii < 0 || jj < 0 || kk < 0 || ii >= n || jj >= n || kk >= n) continue;
                    A.ci[p] = (int)((kk * n + jj) * n + ii);
                    A.v[p] = -w[(dz + 1) * 9 + (dy + 1) * 3 + (dx + 1)];
                    ++p;
                }
    }
}

// Binary system file (examples/test/mtx_gen.cpp:116-146, io/detail/reader.inl):
// u32 nrows, u32 nnz, u32 row[nrows+1], u32 col[nnz], f64 val[nnz],
// f64 b[nrows] (optional), f64 x[nrows] (optional).
bool read_bin(const std::string &path, HostCsr &A, std::vector<double> &b, std::vector<double> &x) {
    FILE *f = fopen(path.c_str(), "rb");
    if (!f) return false;
    uint32_t n = 0, nnz = 0;
    bool ok = fread(&n, 4, 1, f) == 1 && fread(&nnz, 4, 1, f) == 1;
    std::vector<uint32_t> rp(n + 1), ci(nnz);
    ok = ok && fread(rp.data(), 4, n + 1, f) == n + 1 && fread(ci.data(), 4, nnz, f) == nnz;
    A.n = A.ncols = n;
    A.rp.assign(rp.begin(), rp.end());
    A.ci.assign(ci.begin(), ci.end());
    A.v.resize(nnz);
    ok = ok && fread(A.v.data(), 8, nnz, f) == nnz;
    b.resize(n);
    x.resize(n);
    if (fread(b.data(), 8, n, f) != n) b.clear();
    else if (fread(x.data(), 8, n, f) != n) x.clear();
    fclose(f);
    return ok;
}

bool write_bin(const std::string &path, const HostCsr &A, const double *b, const double *x) {
    FILE *f = fopen(path.c_str(), "wb");
    if (!f) return false;
    uint32_t n = (uint32_t)A.n, nnz = (uint32_t)A.nnz();
    fwrite(&n, 4, 1, f);
    fwrite(&nnz, 4, 1, f);
    std::vector<uint32_t> rp(A.rp.begin(), A.rp.end()), ci(A.ci.begin(), A.ci.end());
    fwrite(rp.data(), 4, n + 1, f);
    fwrite(ci.data(), 4, nnz, f);
    fwrite(A.v.data(), 8, nnz, f);
    if (b) fwrite(b, 8, n, f);
    if (b && x) fwrite(x, 8, n, f);
    fclose(f);
    return true;
}

}  // namespace xamg
