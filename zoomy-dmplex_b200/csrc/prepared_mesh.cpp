// Mesh preparation for the device layout (host C++).
//
// Compiled with plain IEEE double arithmetic (-ffp-contract=off, no FMA) so
// the least-squares weights are bit-identical to a straightforward evaluation
// of LeastSquaresGradient::Setup (Gradient.hpp:205-298).
#include "prepared_mesh.h"

#include <algorithm>
#include <cfloat>
#include <cmath>
#include <numeric>

namespace zsme {

namespace {

// Position along a Hilbert curve of order 16 (65536 x 65536 grid).
uint64_t hilbert_d(uint32_t x, uint32_t y) {
    const uint32_t n = 1u << 16;
    uint64_t d = 0;
    for (uint32_t s = n / 2; s > 0; s /= 2) {
        const uint32_t rx = (x & s) > 0;
        const uint32_t ry = (y & s) > 0;
        d += (uint64_t)s * s * ((3 * rx) ^ ry);
        if (ry == 0) {
            if (rx == 1) {
                x = s - 1 - x;
                y = s - 1 - y;
            }
            std::swap(x, y);
        }
    }
    return d;
}

// Cholesky solve of the normal equations (Gradient.hpp:205-217).
bool solve_spd(int n, std::vector<double>& a, std::vector<double>& b) {
    std::vector<double> L(n * n, 0.0);
    for (int i = 0; i < n; i++) {
        for (int j = 0; j <= i; j++) {
            double sum = 0;
            for (int k = 0; k < j; k++) sum += L[i * n + k] * L[j * n + k];
            if (i == j) {
                double val = a[i * n + i] - sum;
                if (val <= 0) return false;
                L[i * n + j] = std::sqrt(val);
            } else {
                L[i * n + j] = (a[i * n + j] - sum) / L[j * n + j];
            }
        }
    }
    for (int i = 0; i < n; i++) {
        double sum = 0;
        for (int k = 0; k < i; k++) sum += L[i * n + k] * b[k];
        b[i] = (b[i] - sum) / L[i * n + i];
    }
    for (int i = n - 1; i >= 0; i--) {
        double sum = 0;
        for (int k = i + 1; k < n; k++) sum += L[k * n + i] * b[k];
        b[i] = (b[i] - sum) / L[i * n + i];
    }
    return true;
}

}  // namespace

int prepare_mesh(const zsme_mesh& m, PreparedMesh& out) {
    const int C = m.n_cells, F = m.n_faces, K = m.max_faces, D = m.dim;
    if (C <= 0 || F <= 0) return set_error(ZSME_ERR_MESH, "empty mesh");
    if (K < 1 || K > 4) return set_error(ZSME_ERR_MESH, "max_faces must be in [1, 4]");
    if (D != 1 && D != 2) return set_error(ZSME_ERR_MESH, "dim must be 1 or 2");
    if (!m.cell_centroid || !m.cell_volume || !m.cell_faces || !m.face_cells || !m.face_centroid ||
        !m.face_normal || !m.face_bc)
        return set_error(ZSME_ERR_ARG, "null mesh array");
    // ---- validation
    for (int f = 0; f < F; ++f) {
        const int a = m.face_cells[2 * f], b = m.face_cells[2 * f + 1];
        if (a < 0 || a >= C || b < -1 || b >= C || a == b)
            return set_error(ZSME_ERR_MESH, "face " + std::to_string(f) + ": invalid support");
        double area = 0;
        for (int d = 0; d < D; ++d) area += m.face_normal[2 * f + d] * m.face_normal[2 * f + d];
        if (!(std::sqrt(area) > 1e-15))
            return set_error(ZSME_ERR_MESH, "face " + std::to_string(f) + ": zero area");
        if (b >= 0 && m.face_bc[f] != ZSME_FACE_INTERIOR)
            return set_error(ZSME_ERR_MESH, "interior face " + std::to_string(f) + " has a boundary marker");
        if (b < 0 && m.face_bc[f] < ZSME_FACE_NO_CONDITION)
            return set_error(ZSME_ERR_MESH, "boundary face " + std::to_string(f) + ": bad marker");
    }
    std::vector<int> seen(F, 0);
    for (int c = 0; c < C; ++c)
        for (int k = 0; k < K; ++k) {
            const int f = m.cell_faces[(size_t)c * K + k];
            if (f < -1 || f >= F) return set_error(ZSME_ERR_MESH, "cell_faces out of range");
            if (f < 0) continue;
            if (m.face_cells[2 * f] != c && m.face_cells[2 * f + 1] != c)
                return set_error(ZSME_ERR_MESH, "cell " + std::to_string(c) + " lists a face it does not support");
            seen[f]++;
        }
    for (int f = 0; f < F; ++f)
        if (seen[f] != (m.face_cells[2 * f + 1] >= 0 ? 2 : 1))
            return set_error(ZSME_ERR_MESH, "face " + std::to_string(f) + " is not in its cells' cones");

    PreparedMesh& p = out;
    p = PreparedMesh();
    p.dim = D;
    p.C = C;
    p.F = F;
    p.K = K;
    // ---- Hilbert order of the cells
    double lo[2] = {DBL_MAX, DBL_MAX}, hi[2] = {-DBL_MAX, -DBL_MAX};
    for (int c = 0; c < C; ++c)
        for (int d = 0; d < 2; ++d) {
            lo[d] = std::min(lo[d], m.cell_centroid[2 * c + d]);
            hi[d] = std::max(hi[d], m.cell_centroid[2 * c + d]);
        }
    std::vector<uint64_t> key(C);
    for (int c = 0; c < C; ++c) {
        uint32_t q[2];
        for (int d = 0; d < 2; ++d) {
            const double span = hi[d] - lo[d];
            const double u = span > 0 ? (m.cell_centroid[2 * c + d] - lo[d]) / span : 0.0;
            q[d] = (uint32_t)std::min(65535.0, std::max(0.0, std::floor(u * 65535.0)));
        }
        key[c] = hilbert_d(q[0], q[1]);
    }
    p.old_of_new.resize(C);
    std::iota(p.old_of_new.begin(), p.old_of_new.end(), 0);
    std::stable_sort(p.old_of_new.begin(), p.old_of_new.end(), [&](int a, int b) { return key[a] < key[b]; });
    p.new_of_old.resize(C);
    for (int c = 0; c < C; ++c) p.new_of_old[p.old_of_new[c]] = c;
    // ---- faces by their lowest new cell
    std::vector<int> fo(F);
    std::iota(fo.begin(), fo.end(), 0);
    auto fkey = [&](int f) {
        const int a = p.new_of_old[m.face_cells[2 * f]];
        const int b = m.face_cells[2 * f + 1] >= 0 ? p.new_of_old[m.face_cells[2 * f + 1]] : a;
        return std::min(a, b);
    };
    std::stable_sort(fo.begin(), fo.end(), [&](int a, int b) { return fkey(a) < fkey(b); });
    p.face_old_of_new = fo;
    std::vector<int> fnew(F);
    for (int i = 0; i < F; ++i) fnew[fo[i]] = i;
    p.fn.assign(2 * (size_t)F, 0.0);
    p.fnr.assign(2 * (size_t)F, 0.0);
    p.fc.assign(2 * (size_t)F, 0.0);
    p.farea.assign(F, 0.0);
    p.face_L.assign(F, -1);
    p.face_R.assign(F, -1);
    p.face_bc.assign(F, ZSME_FACE_INTERIOR);
    for (int i = 0; i < F; ++i) {
        const int f = fo[i];
        p.face_L[i] = p.new_of_old[m.face_cells[2 * f]];
        p.face_R[i] = m.face_cells[2 * f + 1] >= 0 ? p.new_of_old[m.face_cells[2 * f + 1]] : -1;
        p.face_bc[i] = m.face_cells[2 * f + 1] >= 0 ? ZSME_FACE_INTERIOR : m.face_bc[f];
        double area = 0;
        for (int d = 0; d < D; ++d) area += m.face_normal[2 * f + d] * m.face_normal[2 * f + d];
        area = std::sqrt(area);
        p.farea[i] = area;
        for (int d = 0; d < D; ++d) p.fn[(size_t)d * F + i] = m.face_normal[2 * f + d] / area;
        for (int d = 0; d < 2; ++d) {
            p.fnr[(size_t)d * F + i] = m.face_normal[2 * f + d];
            p.fc[(size_t)d * F + i] = m.face_centroid[2 * f + d];
        }
    }
    // ---- per-cell slots
    const size_t KC = (size_t)K * C;
    p.slot_nbr.assign(KC, -2);
    p.slot_meta.assign(KC, 0);
    p.slot_face.assign(KC, -1);
    p.slot_dx.assign(2 * KC, 0.0);
    p.slot_w.assign(2 * KC, 0.0);
    p.vol.assign(C, 0.0);
    p.rc.assign(C, DBL_MAX);
    p.order.assign(C, 0);
    for (int c = 0; c < C; ++c) {
        const int o = p.old_of_new[c];
        p.vol[c] = m.cell_volume[o];
        const double* xc = &m.cell_centroid[2 * o];
        // neighbours in cone order for the least-squares system
        std::vector<int> nb_slot, nb_cell;
        std::vector<std::vector<double>> basis;
        for (int k = 0; k < K; ++k) {
            const int f = m.cell_faces[(size_t)o * K + k];
            if (f < 0) continue;
            const size_t s = (size_t)k * C + c;
            const int L = m.face_cells[2 * f], R = m.face_cells[2 * f + 1];
            const bool isL = (L == o);
            const int other = isL ? R : L;
            int nslot = 0;
            if (other >= 0) {
                for (int kk = 0; kk < K; ++kk)
                    if (m.cell_faces[(size_t)other * K + kk] == f) nslot = kk;
            }
            const int bc = other >= 0 ? ZSME_FACE_INTERIOR : m.face_bc[f];
            p.slot_face[s] = fnew[f];
            p.slot_nbr[s] = other >= 0 ? p.new_of_old[other] : -1;
            p.slot_meta[s] = nslot | ((isL ? 1 : 0) << 2) | ((bc + 2) << 3);
            const double* xf = &m.face_centroid[2 * f];
            for (int d = 0; d < 2; ++d) p.slot_dx[((size_t)k * 2 + d) * C + c] = xf[d] - xc[d];
            double d2 = 0.0;
            for (int d = 0; d < D; ++d) {
                const double dd = xc[d] - xf[d];
                d2 += dd * dd;
            }
            const double dist = std::sqrt(d2);
            if (dist < p.rc[c]) p.rc[c] = dist;
            if (other >= 0) {
                if (std::find(nb_cell.begin(), nb_cell.end(), other) != nb_cell.end()) continue;
                nb_cell.push_back(other);
                nb_slot.push_back(k);
                std::vector<double> b;
                for (int d = 0; d < D; ++d) b.push_back(m.cell_centroid[2 * other + d] - xc[d]);
                basis.push_back(b);
            }
        }
        std::vector<double> ata(D * D, 0.0);
        for (auto& b : basis)
            for (int i = 0; i < D; ++i)
                for (int j = 0; j < D; ++j) ata[i * D + j] += b[i] * b[j];
        for (size_t q = 0; q < basis.size(); ++q) {
            std::vector<double> rhs = basis[q], sys = ata;
            const bool ok = solve_spd(D, sys, rhs);
            for (int d = 0; d < D; ++d) p.slot_w[((size_t)nb_slot[q] * 2 + d) * C + c] = ok ? rhs[d] : 0.0;
        }
        // accumulation order: slots by increasing original face id
        int ks[4] = {0, 1, 2, 3};
        std::stable_sort(ks, ks + K, [&](int a, int b) {
            const int fa = m.cell_faces[(size_t)o * K + a], fb = m.cell_faces[(size_t)o * K + b];
            const long long ka = fa < 0 ? (long long)F + a : fa, kb = fb < 0 ? (long long)F + b : fb;
            return ka < kb;
        });
        int code = 0;
        for (int j = 0; j < K; ++j) code |= ks[j] << (2 * j);
        p.order[c] = code;
    }
    p.n_inst = 1;
    p.inst_cell_off = {0, C};
    p.inst_face_off = {0, F};
    // cells left out of the CFL minimum: no distance constrains them
    if (m.cell_cfl_skip)
        for (int c = 0; c < C; ++c)
            if (m.cell_cfl_skip[p.old_of_new[c]]) p.rc[c] = DBL_MAX;
    return ZSME_OK;
}

int build_tiles(const PreparedMesh& p, int max_faces, FaceTiles& t) {
    const int C = p.C, F = p.F, K = p.K;
    if (max_faces < 2 * K) return set_error(ZSME_ERR_ARG, "tile_faces must be at least twice the face slots");
    t = FaceTiles();
    // faces owned by each cell: those whose lowest cell it is (contiguous runs)
    std::vector<int> own(C, 0);
    for (int f = 0; f < F; ++f) {
        const int L = p.face_L[f], R = p.face_R[f];
        const int lo = R >= 0 ? std::min(L, R) : L;
        if (f > 0) {
            const int pL = p.face_L[f - 1], pR = p.face_R[f - 1];
            if ((pR >= 0 ? std::min(pL, pR) : pL) > lo) return set_error(ZSME_ERR_MESH, "faces not sorted by lowest cell");
        }
        own[lo]++;
    }
    t.cell_off.push_back(0);
    t.face_off.push_back(0);
    t.in_off.push_back(0);
    t.ord_lf.assign((size_t)K * C, -1);
    std::vector<int> in_lf;  // local index of each incoming face of the current tile, per cell slot
    int c0 = 0, f0 = 0;
    while (c0 < C) {
        // grow the tile while its faces fit
        int c = c0, nown = 0, nin = 0;
        while (c < C) {
            int in_c = 0;
            for (int k = 0; k < K; ++k) {
                const int nb = p.slot_nbr[(size_t)k * C + c];
                if (nb >= 0 && nb < c0) in_c++;
            }
            if (c > c0 && nown + nin + own[c] + in_c > max_faces) break;
            nown += own[c];
            nin += in_c;
            ++c;
        }
        const int c1 = c;
        // local face indices: owned faces first (face order), then incoming ones
        int j = 0;
        for (int cc = c0; cc < c1; ++cc) {
            int lf_slot[4] = {-1, -1, -1, -1};
            for (int k = 0; k < K; ++k) {
                const size_t s = (size_t)k * C + cc;
                const int f = p.slot_face[s];
                if (f < 0) continue;
                const int nb = p.slot_nbr[s];
                if (nb >= 0 && nb < c0) {
                    t.in_faces.push_back(f);
                    lf_slot[k] = nown + j++;
                } else {
                    if (f < f0 || f >= f0 + nown) return set_error(ZSME_ERR_MESH, "tile face outside its range");
                    lf_slot[k] = f - f0;
                }
            }
            const int ord = p.order[cc];
            for (int q = 0; q < K; ++q) {
                const int k = (ord >> (2 * q)) & 3;
                const size_t s = (size_t)k * C + cc;
                if (lf_slot[k] < 0) continue;
                const int meta = p.slot_meta[s];
                const bool bc_none = p.slot_nbr[s] < 0 && ((meta >> 3) - 2) < 0;
                if (bc_none) continue;   // exterior face without a condition: no flux
                t.ord_lf[(size_t)q * C + cc] = (lf_slot[k] << 1) | ((meta >> 2) & 1);
            }
        }
        if (j != nin) return set_error(ZSME_ERR_MESH, "incoming face count mismatch");
        t.max_faces = std::max(t.max_faces, nown + nin);
        f0 += nown;
        c0 = c1;
        t.cell_off.push_back(c0);
        t.face_off.push_back(f0);
        t.in_off.push_back((int)t.in_faces.size());
        t.n++;
    }
    if (f0 != F) return set_error(ZSME_ERR_MESH, "tiles do not cover the faces");
    return ZSME_OK;
}

int concat_meshes(std::vector<PreparedMesh>& parts, PreparedMesh& out) {
    if (parts.empty()) return set_error(ZSME_ERR_ARG, "no instances");
    const int K = parts[0].K, D = parts[0].dim;
    long long Ct = 0, Ft = 0;
    for (auto& p : parts) {
        if (p.K != K || p.dim != D) return set_error(ZSME_ERR_MESH, "instances differ in dimension or max_faces");
        Ct += p.C;
        Ft += p.F;
    }
    if (Ct > 0x7fffffffLL || Ft > 0x7fffffffLL) return set_error(ZSME_ERR_LIMIT, "ensemble exceeds 2^31 cells/faces");
    const int C = (int)Ct, F = (int)Ft, n = (int)parts.size();
    PreparedMesh& o = out;
    o = PreparedMesh();
    o.dim = D;
    o.K = K;
    o.C = C;
    o.F = F;
    o.n_inst = n;
    o.old_of_new.resize(C);
    o.slot_nbr.resize((size_t)K * C);
    o.slot_meta.resize((size_t)K * C);
    o.slot_face.resize((size_t)K * C);
    o.slot_dx.resize((size_t)2 * K * C);
    o.slot_w.resize((size_t)2 * K * C);
    o.vol.resize(C);
    o.rc.resize(C);
    o.order.resize(C);
    o.fn.resize(2 * (size_t)F);
    o.fc.resize(2 * (size_t)F);
    o.fnr.resize(2 * (size_t)F);
    o.farea.resize(F);
    o.face_L.resize(F);
    o.face_R.resize(F);
    o.face_bc.resize(F);
    o.cell_inst.resize(C);
    o.face_inst.resize(F);
    o.inst_cell_off.assign(n + 1, 0);
    o.inst_face_off.assign(n + 1, 0);
    int coff = 0, foff = 0;
    for (int i = 0; i < n; ++i) {
        PreparedMesh& p = parts[i];
        o.inst_cell_off[i] = coff;
        o.inst_face_off[i] = foff;
        for (int c = 0; c < p.C; ++c) {
            const int g = coff + c;
            o.old_of_new[g] = p.old_of_new[c];
            o.vol[g] = p.vol[c];
            o.rc[g] = p.rc[c];
            o.order[g] = p.order[c];
            o.cell_inst[g] = i;
            for (int k = 0; k < K; ++k) {
                const size_t s = (size_t)k * p.C + c, t = (size_t)k * C + g;
                const int nb = p.slot_nbr[s], fa = p.slot_face[s];
                o.slot_nbr[t] = nb >= 0 ? nb + coff : nb;
                o.slot_face[t] = fa >= 0 ? fa + foff : fa;
                o.slot_meta[t] = p.slot_meta[s];
                for (int d = 0; d < 2; ++d) {
                    o.slot_dx[((size_t)k * 2 + d) * C + g] = p.slot_dx[((size_t)k * 2 + d) * p.C + c];
                    o.slot_w[((size_t)k * 2 + d) * C + g] = p.slot_w[((size_t)k * 2 + d) * p.C + c];
                }
            }
        }
        for (int f = 0; f < p.F; ++f) {
            const int g = foff + f;
            o.farea[g] = p.farea[f];
            o.face_L[g] = p.face_L[f] + coff;
            o.face_R[g] = p.face_R[f] >= 0 ? p.face_R[f] + coff : -1;
            o.face_bc[g] = p.face_bc[f];
            o.face_inst[g] = i;
            for (int d = 0; d < 2; ++d) {
                o.fn[(size_t)d * F + g] = p.fn[(size_t)d * p.F + f];
                o.fc[(size_t)d * F + g] = p.fc[(size_t)d * p.F + f];
                o.fnr[(size_t)d * F + g] = p.fnr[(size_t)d * p.F + f];
            }
        }
        coff += p.C;
        foff += p.F;
        p = PreparedMesh();  // release the part
    }
    o.inst_cell_off[n] = coff;
    o.inst_face_off[n] = foff;
    return ZSME_OK;
}

}  // namespace zsme
