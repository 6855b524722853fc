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
#include <cstdint>

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


// ---------------------------------------------------------------------------
// Channel with a cube (examples/common/generator/channel_with_cube.inl with
// its geometry lame.inl): a 7-point operator on a curvilinear grid of a
// channel (periodic in x and z, walls at y = 0 and y = ny) around a solid
// block.  The grid lines come from a polynomial index map followed by a
// piecewise-cubic spline per direction; the Lame coefficients H1, H2, H3 are
// central differences of those maps.  The tables below (grid sizes, block
// bounds, index maps, spline breakpoints and coefficients of the three grid
// scales) are the reference's data, restated so that the same matrices come
// out; everything else is this file's own code.
namespace {

struct SplinePiece {
    double below;  // the piece applies to indices < below (the last: any)
    double a[4];   // a0 + a1 s + a2 s^2 + a3 s^3
};

const SplinePiece kSplineX1[] = {
    {14, {1.396162377508623, 2.39973900862267, 0.4213672254912018, 0.03526915777851145}},
    {24, {-3.307327090264011, -7.600783718893908, -6.666310657693695, -1.639149241623937}},
    {46, {-0.2168199280894425, 1.054198523421452, 1.413131074030182, 0.8749086296590155}},
    {56, {0.1785684516356735, 3.426528801772148, 6.157791630731574, 4.038015667459944}},
    {88, {0.0, 1.610279383056608, 0.0, -2.921086861223202}},
    {98, {-0.1785684516356735, 3.426528801772148, -6.157791630731574, 4.038015667459944}},
    {120, {0.2168199280894425, 1.054198523421452, -1.413131074030183, 0.8749086296590157}},
    {130, {3.307327090264012, -7.600783718893908, 6.666310657693695, -1.639149241623937}},
    {1e300, {-1.396162377508623, 2.39973900862267, -0.4213672254912018, 0.03526915777851145}},
};
const SplinePiece kSplineX2[] = {
    {9, {1.663364261477938, 2.763116308992502, 0.5920931128840505, 0.06318801187864154}},
    {42, {-1.114914960494785, -2.080698526151822, -2.222903782988859, -0.4821264969997728}},
    {70, {-0.4236400477834716, 0.1334790192104974, 0.1411254004985186, 0.3592143418872756}},
    {90, {0.1851416166778065, 3.786169005978167, 7.446505374033857, 5.229467657577501}},
    {150, {0.0, 1.752459555086567, 0.0, -3.859087619448435}},
    {170, {-0.1851416166778064, 3.786169005978166, -7.446505374033855, 5.229467657577499}},
    {198, {0.4236400477834715, 0.1334790192104982, -0.1411254004985194, 0.3592143418872759}},
    {231, {1.114914960494784, -2.080698526151822, 2.222903782988859, -0.4821264969997728}},
    {1e300, {-1.663364261477938, 2.763116308992505, -0.5920931128840512, 0.0631880118786417}},
};
const SplinePiece kSplineX3[] = {
    {15, {1.031662508857209, 1.969399191066359, 0.2286523094234516, 9.341705522873112e-4}},
    {65, {-0.7588674138101876, -1.206056260460024, -1.648541921732235, -0.368971630917371}},
    {105, {-0.5215911974286817, -0.4253232006982945, -0.7922345627386506, -0.05590590211357671}},
    {132, {0.2395985844288585, 4.141815490446947, 8.342042819551832, 6.033612352746744}},
    {228, {0.0, 1.693096447267712, 0.0, -3.439323928921869}},
    {255, {-0.2395985844288585, 4.141815490446947, -8.342042819551834, 6.033612352746745}},
    {295, {0.5215911974286818, -0.4253232006982945, 0.7922345627386508, -0.05590590211357682}},
    {345, {0.7588674138101876, -1.206056260460024, 1.648541921732235, -0.368971630917371}},
    {1e300, {-1.03166250885721, 1.969399191066359, -0.228652309423452, 9.341705522873667e-4}},
};
const SplinePiece kSplineY1[] = {
    {10, {0.0, 0.4500000000000001, -0.2935533747052894, 6.708531575913051}},
    {38, {0.03430441990176908, -0.2280167698232014, 4.173380638247565, -3.10120586429714}},
    {48, {-2.563649298895133, 10.37415873036821, -10.24901194500876, 3.438502513535689}},
    {64, {-0.008557016802147377, 2.708881884089249, -2.583735098729805, 0.8834102314427034}},
    {87, {5.052109496470486, -7.509771652326646, 4.294204781550124, -0.6597173057995884}},
    {98, {7.504547694864687, -10.6845712464721, 5.664181874766423, -0.856773023310955}},
    {1e300, {-28.34061977576933, 28.12523413526699, -8.342364428417605, 0.8282250281999057}},
};
const SplinePiece kSplineY2[] = {
    {20, {0.0, 0.5, -0.5684921832901438, 5.517772964909718}},
    {59, {0.06233578376582055, -0.4689042295569277, 4.451499809217404, -3.151924491966832}},
    {74, {-2.185198059852231, 8.717375665526223, -8.064105321035434, 2.531927715361443}},
    {88, {-2.21918495246137, 8.81933634335364, -8.166065998862852, 2.565914607970583}},
    {120, {4.742597325172884, -7.531522690118807, 4.634803111498467, -0.7746285330177924}},
    {153, {1.635341021829459, -2.908803297044359, 2.342369691044022, -0.3956848463868132}},
    {1e300, {-30.09333727085763, 29.55298527669742, -8.728242912540622, 0.8628046865218802}},
};
const SplinePiece kSplineY3[] = {
    {20, {0.0, 0.8675000000000002, -2.635398381455771, 20.00101762126424}},
    {90, {0.01600837036955505, 0.3248684456798112, 3.495748365455494, -3.090747028787434}},
    {120, {-1.497835823305939, 7.37167970490478, -7.438346686641689, 2.564502805042847}},
    {143, {-0.257719998070995, 3.651332229199951, -3.717999210936858, 1.324386979807903}},
    {180, {4.797985956621731, -7.837124154581934, 4.984025212216816, -0.8727526686501045}},
    {233, {0.7330112214661275, -1.492467642278255, 1.683089053788552, -0.3002930195533108}},
    {1e300, {-28.27470371382332, 27.801962358161, -8.17823727456962, 0.806239939703357}},
};

struct ChannelGrid {
    i64 nx, ny, nz;
    i64 bx0, bx1, by0, by1, bz0, bz1;   // solid block [b0, b1) per direction
    double mapx[4], mapy[4];            // index maps (cubic polynomials)
    const SplinePiece *sx, *sy;
    int nsx, nsy;
    double hx, hy, hz;

    explicit ChannelGrid(int scale) {
        // per scale: sizes, block, index-map coefficients (highest first as
        // written: c3, c2, c1, c0)
        if (scale == 1) {
            set(144, 112, 144, 46, 98, 0, 48, 46, 98);
            setmap(mapx, 1.0 / 527436.0, -216.0 / 527436.0, 25019.0 / 527436.0, -2.0);
            setmap(mapy, 0.0, 1.0 / 6720.0, 92.0 / 6720.0, 0.0);
            sx = kSplineX1; nsx = 9; sy = kSplineY1; nsy = 7;
        } else if (scale == 2) {
            set(240, 168, 240, 70, 170, 0, 74, 70, 170);
            setmap(mapx, 1.0 / 1785000.0, -360.0 / 1785000.0, 58550.0 / 1785000.0, -2.0);
            setmap(mapy, 0.0, 209.0 / 2921520.0, 24014.0 / 2921520.0, 0.0);
            sx = kSplineX2; nsx = 9; sy = kSplineY2; nsy = 7;
        } else if (scale == 3) {
            set(360, 252, 360, 105, 255, 0, 120, 105, 255);
            setmap(mapx, 2.0 / 12048750.0, -1080.0 / 12048750.0, 263475.0 / 12048750.0, -2.0);
            setmap(mapy, 0.0, 13.0 / 332640.0, 1212.0 / 332640.0, 0.0);
            sx = kSplineX3; nsx = 9; sy = kSplineY3; nsy = 7;
        } else {
            throw Error("channel_with_cube: grid scale must be 1, 2 or 3", 2);
        }
        hx = 4.0 / nx;   // channel 4 x 3.4 x 4
        hy = 3.4 / ny;
        hz = 4.0 / nz;
    }
    void set(i64 x, i64 y, i64 z, i64 x0, i64 x1, i64 y0, i64 y1, i64 z0, i64 z1) {
        nx = x; ny = y; nz = z;
        bx0 = x0; bx1 = x1; by0 = y0; by1 = y1; bz0 = z0; bz1 = z1;
    }
    static void setmap(double *m, double c3, double c2, double c1, double c0) {
        m[0] = c0; m[1] = c1; m[2] = c2; m[3] = c3;
    }
    // a0 + a1 s + a2 s^2 + a3 s^3, summed in that order with pow() terms
    static double cubic(const double *a, double s) {
        double v = 0.0;
        for (int p = 0; p < 4; ++p) v += a[p] * std::pow(s, p);
        return v;
    }
    static const double *piece(const SplinePiece *t, int cnt, double idx) {
        for (int q = 0; q < cnt - 1; ++q)
            if (idx < t[q].below) return t[q].a;
        return t[cnt - 1].a;
    }
    // coordinate of the grid position x (x and z directions, y direction)
    double line_xz(double x) const {
        const double ic = x / hx;
        return cubic(piece(sx, nsx, ic), cubic(mapx, ic));
    }
    double line_y(double y) const {
        const double jc = y / hy;
        return cubic(piece(sy, nsy, jc), cubic(mapy, jc));
    }
    // Lame coefficients: central differences of the maps over 0.02 h
    double h1(double x) const { return (line_xz(x + 0.01 * hx) - line_xz(x - 0.01 * hx)) / (0.02 * hx); }
    double h2(double y) const { return (line_y(y + 0.01 * hy) - line_y(y - 0.01 * hy)) / (0.02 * hy); }
    double h3(double z) const { return (line_xz(z + 0.01 * hz) - line_xz(z - 0.01 * hz)) / (0.02 * hz); }
    double H(double x, double y, double z) const { return h1(x) * h2(y) * h3(z); }
    // H at the cell centre and at the low x, y, z faces of cell (i, j, k)
    double Hc(i64 i, i64 j, i64 k) const { return H((i + 0.5) * hx, (j + 0.5) * hy, (k + 0.5) * hz); }
    double Hx(i64 i, i64 j, i64 k) const { return H(i * hx, (j + 0.5) * hy, (k + 0.5) * hz); }
    double Hy(i64 i, i64 j, i64 k) const { return H((i + 0.5) * hx, j * hy, (k + 0.5) * hz); }
    double Hz(i64 i, i64 j, i64 k) const { return H((i + 0.5) * hx, (j + 0.5) * hy, k * hz); }
    // indices as the reference evaluates them: unsigned, so -1 wraps to a
    // huge value (outside every range)
    bool solid(uint64_t i, uint64_t j, uint64_t k) const {
        return i >= (uint64_t)bx0 && i < (uint64_t)bx1 && j >= (uint64_t)by0 && j < (uint64_t)by1 &&
               k >= (uint64_t)bz0 && k < (uint64_t)bz1;
    }
    bool ywall(uint64_t j) const { return j >= (uint64_t)ny; }
};

// The reference's pseudo-random stream (src/misc/rand.h): a 32-bit xorshift of
// i + 1 (shifts 13, 17, 5) fed to one linear-congruential step (1664525,
// 1013904223) in 32-bit two's-complement arithmetic, mapped to (0, 1] as
// 0.5 (1 + v / INT_MAX).  i is taken modulo 2^32, as there.
double stream_value(uint64_t i) {
    uint32_t s = (uint32_t)i + 1u;
    s ^= s << 13;
    s ^= s >> 17;
    s ^= s << 5;
    const uint32_t g = 1664525u * s + 1013904223u;
    const int32_t v = (int32_t)g;
    return 0.5 * (1.0 + (double)v / 2147483647.0);
}

}  // namespace

// Channel-with-cube system of grid scale 1..3: the operator (rows x
// lexicographic, diagonal first, then the bottom, south, west, east, north,
// top neighbours that exist) and, for nv columns, the right-hand side: 1
// everywhere (const_rhs) or the discrete divergence of pseudo-random face
// velocities 0.1 * stream(face * nv + column).  The last row is an identity
// row (its other entries kept at 0) with right-hand side 0 in the divergence
// form.
void gen_channel_cube(int scale, bool const_rhs, int nv, HostCsr &A, std::vector<double> &b) {
    const ChannelGrid g(scale);
    const i64 nx = g.nx, ny = g.ny, nz = g.nz, N = nx * ny * nz;
    A.n = A.ncols = N;
    // the couplings of row r that exist, in row order (b, s, w, e, n, t); a
    // solid cell has none
    auto links = [&](uint64_t i, uint64_t j, uint64_t k, bool *open) {
        const bool fluid = !g.solid(i, j, k);
        open[0] = fluid && !g.solid(i, j, k - 1);
        open[1] = fluid && !g.solid(i, j - 1, k) && !g.ywall(j - 1);
        open[2] = fluid && !g.solid(i - 1, j, k);
        open[3] = fluid && !g.solid(i + 1, j, k);
        open[4] = fluid && !g.solid(i, j + 1, k) && !g.ywall(j + 1);
        open[5] = fluid && !g.solid(i, j, k + 1);
    };
    A.rp.assign(N + 1, 0);
    for (i64 r = 0; r < N; ++r) {
        bool open[6];
        links(r % nx, (r / nx) % ny, r / (nx * ny), open);
        int c = 1;
        for (bool o : open) c += o;
        A.rp[r + 1] = A.rp[r] + c;
    }
    A.ci.assign(A.rp[N], 0);
    A.v.assign(A.rp[N], 0.0);
#pragma omp parallel for schedule(dynamic, 4096)
    for (i64 r = 0; r < N; ++r) {
        const uint64_t i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
        bool open[6];
        links(i, j, k, open);
        int *cols = &A.ci[A.rp[r]];
        double *vals = &A.v[A.rp[r]];
        const int cnt = A.rp[r + 1] - A.rp[r];
        cols[0] = (int)r;
        vals[0] = 0.0;
        if (!g.solid(i, j, k)) {
            const double q_e = (g.Hx(i + 1, j, k) / std::pow(g.h1((i + 1) * g.hx), 2.)) / (g.hx * g.hx);
            const double q_w = (g.Hx(i, j, k) / std::pow(g.h1(i * g.hx), 2.)) / (g.hx * g.hx);
            const double q_n = (g.Hy(i, j + 1, k) / std::pow(g.h2((j + 1) * g.hy), 2.)) / (g.hy * g.hy);
            const double q_s = (g.Hy(i, j, k) / std::pow(g.h2(j * g.hy), 2.)) / (g.hy * g.hy);
            const double q_t = (g.Hz(i, j, k + 1) / std::pow(g.h3((k + 1) * g.hz), 2.)) / (g.hz * g.hz);
            const double q_b = (g.Hz(i, j, k) / std::pow(g.h3(k * g.hz), 2.)) / (g.hz * g.hz);
            const double q[6] = {q_b, q_s, q_w, q_e, q_n, q_t};
            const i64 nb[6] = {(i64)(((k - 1 + nz) % nz) * nx * ny + j * nx + i), (i64)(k * nx * ny + (j - 1) * nx + i),
                               (i64)(k * nx * ny + j * nx + (i - 1 + nx) % nx), (i64)(k * nx * ny + j * nx + (i + 1) % nx),
                               (i64)(k * nx * ny + (j + 1) * nx + i), (i64)(((k + 1) % nz) * nx * ny + j * nx + i)};
            int p = 1;
            for (int d = 0; d < 6; ++d) {
                if (!open[d]) continue;
                vals[0] += q[d];
                vals[p] = -q[d];
                cols[p] = (int)nb[d];
                ++p;
            }
        } else {
            vals[0] = 1.0;
        }
        if (r == N - 1) {
            vals[0] = 1.0;
            for (int q = 1; q < cnt; ++q) vals[q] = 0.0;
        }
        // scaled by 1/H_c and then by H_c hx hy hz, two roundings as there
        const double hc = g.Hc(i, j, k);
        const double s1 = 1. / hc, s2 = hc * g.hx * g.hy * g.hz;
        for (int q = 0; q < cnt; ++q) vals[q] *= s1;
        for (int q = 0; q < cnt; ++q) vals[q] *= s2;
    }
    b.assign((size_t)N * nv, 1.0);
    if (const_rhs) return;
    const double ihx = 1. / g.hx, ihy = 1. / g.hy, ihz = 1. / g.hz;
#pragma omp parallel for schedule(dynamic, 4096)
    for (i64 r = 0; r < N; ++r) {
        const uint64_t i = r % nx, j = (r / nx) % ny, k = r / (nx * ny);
        const double Hc = g.Hc(i, j, k);
        const double w_ = g.Hx(i, j, k) / g.h1(i * g.hx), e_ = g.Hx(i + 1, j, k) / g.h1((i + 1) * g.hx);
        const double s_ = g.Hy(i, j, k) / g.h2(j * g.hy), n_ = g.Hy(i, j + 1, k) / g.h2((j + 1) * g.hy);
        const double b_ = g.Hz(i, j, k) / g.h3(k * g.hz), t_ = g.Hz(i, j, k + 1) / g.h3((k + 1) * g.hz);
        // face numbering of the three velocity components
        const uint64_t fe = k * ny * (nx + 1) + j * (nx + 1) + i + 1, fw = fe - 1;
        const uint64_t fn = k * (ny + 1) * nx + (j + 1) * nx + i, fs = k * (ny + 1) * nx + j * nx + i;
        const uint64_t ft = (k + 1) * ny * nx + j * nx + i, fb = k * ny * nx + j * nx + i;
        for (int c = 0; c < nv; ++c) {
            auto vel = [&](uint64_t f) { return 0.1 * stream_value(f * (uint64_t)nv + (uint64_t)c); };
            double v = -((e_ * vel(fe) - w_ * vel(fw)) * ihx + (n_ * vel(fn) - s_ * vel(fs)) * ihy +
                         (t_ * vel(ft) - b_ * vel(fb)) * ihz) /
                       Hc;
            if (r == N - 1) v = 0.;
            b[(size_t)r * nv + c] = v;
        }
    }
}

}  // namespace xamg
