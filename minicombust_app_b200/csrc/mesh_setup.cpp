// Host-side mesh import and geometry for the B200 flow solver.
//
// Built with FMA contraction off: the geometry formulas are evaluated in the
// operation order of the reference constructor (FlowSolver.hpp:253-398), so
// face areas, normals, centres, interpolation weights and cell volumes equal
// the reference's bit for bit.
#include "mesh_setup.h"

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>

#include "minicombust_flow.h"

namespace mcb {

namespace {

struct V3 {
    double x, y, z;
};
inline V3 add(V3 a, V3 b) { return {a.x + b.x, a.y + b.y, a.z + b.z}; }
inline V3 sub(V3 a, V3 b) { return {a.x - b.x, a.y - b.y, a.z - b.z}; }
inline V3 scale(V3 a, double s) { return {a.x * s, a.y * s, a.z * s}; }
inline V3 divs(V3 a, double s) { return {a.x / s, a.y / s, a.z / s}; }
inline double dot(V3 a, V3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
inline double mag(V3 a) { return std::sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }
inline V3 cross(V3 a, V3 b) { return {a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x}; }
inline double cosangle(V3 a, V3 b) { return dot(a, b) / (mag(a) * mag(b)); }
inline V3 ld(const double *p, uint64_t i) { return {p[3 * i], p[3 * i + 1], p[3 * i + 2]}; }

// CUBE_FACE_VERTEX_MAP (Mesh.hpp:20-28), vertex order A..H = 0..7.
const int kFaceVertex[6][4] = {{0, 1, 2, 3}, {4, 5, 6, 7}, {0, 2, 4, 6}, {1, 3, 5, 7}, {0, 1, 4, 5}, {2, 3, 6, 7}};

} // namespace

int build_host_mesh(const mc_mesh_view *mv, const HostPhysics &hp, HostMesh &hm, std::string &err)
{
    const uint64_t N64 = mv->cells, F64 = mv->faces;
    if (N64 == 0 || F64 == 0 || N64 + 6 >= (uint64_t)INT32_MAX || F64 >= (uint64_t)INT32_MAX) {
        err = "mesh size out of range (cells and faces must fit in int32)";
        return MC_ERR_MESH;
    }
    if (!mv->points_xyz || !mv->cell_nodes || !mv->face_cells || !mv->cell_faces || !mv->cell_neighbours ||
        !mv->cell_centers) {
        err = "mesh view has a null array";
        return MC_ERR_ARG;
    }
    const int N = (int)N64, F = (int)F64;
    hm.N = N;
    hm.F = F;
    for (int s = 0; s < 6; s++) {
        const uint64_t t = mv->boundary_types[s];
        if (t < 1 || t > 3) {
            err = "boundary_types must be 1 (wall), 2 (inlet) or 3 (outlet)";
            return MC_ERR_MESH;
        }
        hm.btype[s] = (int)t;
        hm.last_bface[s] = -1;
    }
    try {
        hm.fc0.resize(F);
        hm.fc1.resize(F);
        hm.nbr.resize((size_t)6 * N);
        hm.sface.resize((size_t)6 * N);
        hm.col.resize((size_t)6 * N);
        hm.area.assign(F, 0.0);
        hm.lam.assign(F, 0.0);
        hm.rl.assign(F, 0.0);
        hm.S.assign((size_t)3 * F, 0.0);
        hm.xf.assign((size_t)3 * F, 0.0);
        hm.xc.resize((size_t)3 * N);
        hm.vol.resize(N);
        hm.rho.assign(N, hp.density);
    } catch (const std::bad_alloc &) {
        err = "host allocation failed";
        return MC_ERR_NOMEM;
    }
    for (int f = 0; f < F; f++) {
        const uint64_t c0 = mv->face_cells[2 * (size_t)f], c1 = mv->face_cells[2 * (size_t)f + 1];
        if (c0 >= N64 || c1 == c0 || (c1 >= N64 && c1 - N64 >= 6) || (c1 < N64 && c1 < c0)) {
            err = "face " + std::to_string(f) + " has invalid cells";
            return MC_ERR_MESH;
        }
        hm.fc0[f] = (int)c0;
        hm.fc1[f] = (int)c1;
        if (c1 >= N64) {
            const int side = (int)(c1 - N64);
            hm.last_bface[side] = std::max(hm.last_bface[side], f);  // last face in reference order
            if (hm.btype[side] == 3) hm.outlet_faces.push_back(f);
        }
    }
    for (int c = 0; c < N; c++) {
        int faces[6];
        for (int s = 0; s < 6; s++) {
            const uint64_t f = mv->cell_faces[6 * (size_t)c + s];
            if (f >= F64 || (hm.fc0[f] != c && hm.fc1[f] != c)) {
                err = "cell_faces of cell " + std::to_string(c) + " is inconsistent with faces";
                return MC_ERR_MESH;
            }
            faces[s] = (int)f;
            const int other = (hm.fc0[f] == c) ? hm.fc1[f] : hm.fc0[f];
            hm.nbr[(size_t)s * N + c] = (other < N) ? other : -1 - (int)f;
        }
        int sorted[6];
        std::copy(faces, faces + 6, sorted);
        std::sort(sorted, sorted + 6);
        for (int k = 0; k < 6; k++) {
            if (k > 0 && sorted[k] == sorted[k - 1]) {
                err = "cell " + std::to_string(c) + " lists a face twice";
                return MC_ERR_MESH;
            }
            const int f = sorted[k];
            hm.sface[(size_t)k * N + c] = f;
            const int other = (hm.fc0[f] == c) ? hm.fc1[f] : hm.fc0[f];
            hm.col[(size_t)k * N + c] = (other < N) ? other : c;
        }
        for (int d = 0; d < 3; d++) hm.xc[3 * (size_t)c + d] = mv->cell_centers[3 * (size_t)c + d];
    }

    const double *pts = mv->points_xyz;
    const uint64_t P = mv->points;
    // internal faces (FlowSolver.hpp:253-294)
    for (int f = 0; f < F; f++) {
        const int c0 = hm.fc0[f], c1 = hm.fc1[f];
        if (c1 >= N) continue;
        uint64_t ids[4];
        int cnt = 0;
        for (int n0 = 0; n0 < 8; n0++)
            for (int n1 = 0; n1 < 8; n1++)
                if (mv->cell_nodes[8 * (size_t)c0 + n0] == mv->cell_nodes[8 * (size_t)c1 + n1] && cnt < 4)
                    ids[cnt++] = mv->cell_nodes[8 * (size_t)c0 + n0];
        if (cnt != 4 || ids[0] >= P || ids[1] >= P || ids[2] >= P || ids[3] >= P) {
            err = "internal face " + std::to_string(f) + " does not share exactly four nodes";
            return MC_ERR_MESH;
        }
        const V3 n0 = ld(pts, ids[0]), n1 = ld(pts, ids[1]), n2 = ld(pts, ids[2]), n3 = ld(pts, ids[3]);
        const V3 x0 = ld(mv->cell_centers, (uint64_t)c0), x1 = ld(mv->cell_centers, (uint64_t)c1);
        const V3 d01 = sub(x1, x0);
        hm.area[f] = mag(sub(n2, n0)) * mag(sub(n1, n0));
        V3 fc = add(add(add(n0, n1), n2), n3);
        fc = divs(fc, 4.0);
        hm.lam[f] = mag(sub(fc, x0)) / mag(d01);
        V3 S = cross(sub(n2, n0), sub(n1, n0));
        if (dot(S, sub(x1, x0)) < 0) S = scale(S, -1.);
        hm.rl[f] = hm.area[f] / mag(d01) / cosangle(S, d01);
        hm.S[3 * (size_t)f] = S.x;
        hm.S[3 * (size_t)f + 1] = S.y;
        hm.S[3 * (size_t)f + 2] = S.z;
        hm.xf[3 * (size_t)f] = fc.x;
        hm.xf[3 * (size_t)f + 1] = fc.y;
        hm.xf[3 * (size_t)f + 2] = fc.z;
    }
    // cell volumes and boundary faces (FlowSolver.hpp:302-397)
    for (int c = 0; c < N; c++) {
        const uint64_t *cn = mv->cell_nodes + 8 * (size_t)c;
        for (int i = 0; i < 8; i++)
            if (cn[i] >= P) {
                err = "cell " + std::to_string(c) + " references a missing point";
                return MC_ERR_MESH;
            }
        const double width = mag(sub(ld(pts, cn[1]), ld(pts, cn[0])));
        const double height = mag(sub(ld(pts, cn[2]), ld(pts, cn[0])));
        const double length = mag(sub(ld(pts, cn[4]), ld(pts, cn[0])));
        hm.vol[c] = width * height * length;
        const V3 xcell = ld(mv->cell_centers, (uint64_t)c);
        for (int s = 0; s < 6; s++) {
            if (mv->cell_neighbours[6 * (size_t)c + s] < N64) continue;
            const int face = (int)mv->cell_faces[6 * (size_t)c + s];
            if (hm.fc1[face] < N) {
                err = "cell_neighbours marks an internal face of cell " + std::to_string(c) + " as boundary";
                return MC_ERR_MESH;
            }
            const V3 n0 = ld(pts, cn[kFaceVertex[s][0]]), n1 = ld(pts, cn[kFaceVertex[s][1]]);
            const V3 n2 = ld(pts, cn[kFaceVertex[s][2]]), n3 = ld(pts, cn[kFaceVertex[s][3]]);
            hm.lam[face] = 1.0;
            hm.area[face] = mag(sub(n2, n0)) * mag(sub(n1, n0));
            const V3 fc = divs(add(add(add(n0, n1), n2), n3), 4.0);
            V3 S = cross(sub(n2, n0), sub(n1, n0));
            if (dot(S, sub(xcell, fc)) > 0) S = scale(S, -1.);  // outward for every boundary type
            const V3 dcf = sub(fc, xcell);
            hm.rl[face] = hm.area[face] / mag(dcf) / cosangle(S, dcf);
            hm.S[3 * (size_t)face] = S.x;
            hm.S[3 * (size_t)face + 1] = S.y;
            hm.S[3 * (size_t)face + 2] = S.z;
            hm.xf[3 * (size_t)face] = fc.x;
            hm.xf[3 * (size_t)face + 1] = fc.y;
            hm.xf[3 * (size_t)face + 2] = fc.z;
        }
    }
    for (int s = 0; s < 6; s++)
        if (hm.last_bface[s] < 0) {
            err = "boundary side " + std::to_string(s) + " has no faces";
            return MC_ERR_MESH;
        }
    return MC_OK;
}

namespace {

// Breadth-first levels from r over unvisited (global mark 0) cells; returns
// the cells of the last level and the eccentricity.
int bfs_last_level(const HostMesh &hm, const std::vector<int> &deg, int r, std::vector<int> &dist,
                   std::vector<int> &touched, std::vector<int> &last)
{
    const int N = hm.N;
    for (int t : touched) dist[t] = -1;
    touched.clear();
    dist[r] = 0;
    touched.push_back(r);
    int ecc = 0;
    for (size_t head = 0; head < touched.size(); head++) {
        const int u = touched[head];
        ecc = dist[u];
        for (int s = 0; s < 6; s++) {
            const int v = hm.nbr[(size_t)s * N + u];
            if (v >= 0 && dist[v] < 0) {
                dist[v] = dist[u] + 1;
                touched.push_back(v);
            }
        }
    }
    last.clear();
    for (int t : touched)
        if (dist[t] == ecc) last.push_back(t);
    (void)deg;
    return ecc;
}

} // namespace

void rcm_cell_order(const HostMesh &hm, std::vector<int> &order)
{
    const int N = hm.N;
    std::vector<int> deg(N, 0);
    for (int c = 0; c < N; c++)
        for (int s = 0; s < 6; s++) deg[c] += hm.nbr[(size_t)s * N + c] >= 0;
    std::vector<int> by_deg(N);
    for (int c = 0; c < N; c++) by_deg[c] = c;
    std::stable_sort(by_deg.begin(), by_deg.end(), [&](int a, int b) { return deg[a] < deg[b]; });
    std::vector<char> seen(N, 0);
    std::vector<int> dist(N, -1), touched, last, nb;
    order.clear();
    order.reserve(N);
    size_t cand = 0;
    while ((int)order.size() < N) {
        while (seen[by_deg[cand]]) cand++;
        // pseudo-peripheral start (George & Liu): move to a least-degree cell
        // of the last BFS level while the eccentricity grows
        int r = by_deg[cand];
        int ecc = bfs_last_level(hm, deg, r, dist, touched, last);
        for (int sweep = 0; sweep < 8; sweep++) {
            int best = last[0];
            for (int t : last)
                if (deg[t] < deg[best] || (deg[t] == deg[best] && t < best)) best = t;
            const int e2 = bfs_last_level(hm, deg, best, dist, touched, last);
            if (e2 <= ecc) break;
            r = best;
            ecc = e2;
        }
        for (int t : touched) dist[t] = -1;
        touched.clear();
        // Cuthill-McKee sweep of the component
        size_t head = order.size();
        order.push_back(r);
        seen[r] = 1;
        for (; head < order.size(); head++) {
            const int u = order[head];
            nb.clear();
            for (int s = 0; s < 6; s++) {
                const int v = hm.nbr[(size_t)s * N + u];
                if (v >= 0 && !seen[v]) {
                    seen[v] = 1;
                    nb.push_back(v);
                }
            }
            std::sort(nb.begin(), nb.end(), [&](int a, int b) { return deg[a] != deg[b] ? deg[a] < deg[b] : a < b; });
            order.insert(order.end(), nb.begin(), nb.end());
        }
    }
    std::reverse(order.begin(), order.end());
}

int apply_reorder(HostMesh &hm, const std::vector<int> &cell_n2o, std::vector<int> &face_n2o, std::string &err)
{
    const int N = hm.N, F = hm.F;
    if ((int)cell_n2o.size() != N) {
        err = "cell permutation has the wrong length";
        return MC_ERR_ARG;
    }
    std::vector<int> co2n(N, -1), fo2n(F, -1);
    for (int n = 0; n < N; n++) {
        const int o = cell_n2o[n];
        if (o < 0 || o >= N || co2n[o] >= 0) {
            err = "cell permutation is not a permutation";
            return MC_ERR_ARG;
        }
        co2n[o] = n;
    }
    face_n2o.clear();
    face_n2o.reserve(F);
    for (int n = 0; n < N; n++)
        for (int k = 0; k < 6; k++) {
            const int f = hm.sface[(size_t)k * N + cell_n2o[n]];
            if (fo2n[f] < 0) {
                fo2n[f] = (int)face_n2o.size();
                face_n2o.push_back(f);
            }
        }
    if ((int)face_n2o.size() != F) {
        err = "some faces belong to no cell";
        return MC_ERR_MESH;
    }
    auto cell_id = [&](int c) { return c < N ? co2n[c] : c; };  // boundary slots N + side stay
    std::vector<int> fc0(F), fc1(F);
    std::vector<double> area(F), lam(F), rl(F), S(3 * (size_t)F), xf(3 * (size_t)F);
    for (int n = 0; n < F; n++) {
        const int o = face_n2o[n];
        fc0[n] = cell_id(hm.fc0[o]);
        fc1[n] = cell_id(hm.fc1[o]);
        area[n] = hm.area[o];
        lam[n] = hm.lam[o];
        rl[n] = hm.rl[o];
        for (int d = 0; d < 3; d++) {
            S[3 * (size_t)n + d] = hm.S[3 * (size_t)o + d];
            xf[3 * (size_t)n + d] = hm.xf[3 * (size_t)o + d];
        }
    }
    std::vector<int> nbr((size_t)6 * N), sface((size_t)6 * N), col((size_t)6 * N);
    std::vector<double> xc(3 * (size_t)N), vol(N), rho(N);
    for (int n = 0; n < N; n++) {
        const int o = cell_n2o[n];
        for (int k = 0; k < 6; k++) {
            const int v = hm.nbr[(size_t)k * N + o];
            nbr[(size_t)k * N + n] = v >= 0 ? co2n[v] : -1 - fo2n[-1 - v];
            sface[(size_t)k * N + n] = fo2n[hm.sface[(size_t)k * N + o]];
            col[(size_t)k * N + n] = co2n[hm.col[(size_t)k * N + o]];
        }
        for (int d = 0; d < 3; d++) xc[3 * (size_t)n + d] = hm.xc[3 * (size_t)o + d];
        vol[n] = hm.vol[o];
        rho[n] = hm.rho[o];
    }
    for (int &f : hm.outlet_faces) f = fo2n[f];
    for (int s = 0; s < 6; s++) hm.last_bface[s] = fo2n[hm.last_bface[s]];
    hm.fc0.swap(fc0);
    hm.fc1.swap(fc1);
    hm.area.swap(area);
    hm.lam.swap(lam);
    hm.rl.swap(rl);
    hm.S.swap(S);
    hm.xf.swap(xf);
    hm.nbr.swap(nbr);
    hm.sface.swap(sface);
    hm.col.swap(col);
    hm.xc.swap(xc);
    hm.vol.swap(vol);
    hm.rho.swap(rho);
    return MC_OK;
}

// Inlet effective viscosity (FlowSolver.hpp:421-422).
double inlet_effective_viscosity(double mu, double u_in)
{
    const double velmag2 = std::pow(u_in, 2) + std::pow(0.0, 2) + std::pow(0.0, 2);
    return mu + 1.2 * 0.09 * (3.0 / 2.0 * ((0.1 * 0.1) * velmag2)) /
                    ((std::pow(0.09, 0.75) * std::pow((3.0 / 2.0 * ((0.1 * 0.1) * velmag2)), 1.5)) +
                     0.00000000000000000001);
}

} // namespace mcb

// ------------------------------------------------------------ box mesh API

// load_mesh for one flow rank (src/examples/mesh_examples.cpp:120-571): one
// block, cells x-fastest, neighbours as fill_neighbours (:13-118), faces made
// in cell order with the partner-slot trick (:510-561), cell centres as the
// vertex mean (Mesh.hpp:54-67).
extern "C" int mc_mesh_box_create(uint64_t ex, uint64_t ey, uint64_t ez, double lx, double ly, double lz,
                                  mc_mesh_view *out)
{
    if (!out || ex == 0 || ey == 0 || ez == 0) return MC_ERR_ARG;
    memset(out, 0, sizeof(*out));
    const uint64_t px = ex + 1, py = ey + 1, pz = ez + 1;
    const uint64_t N = ex * ey * ez;
    const uint64_t F = (ex + 1) * ey * ez + (ey + 1) * ex * ez + (ez + 1) * ex * ey;
    const uint64_t P = px * py * pz;
    const double dx = lx / (double)ex, dy = ly / (double)ey, dz = lz / (double)ez;
    double *points = new (std::nothrow) double[3 * P];
    uint64_t *cells = new (std::nothrow) uint64_t[8 * N];
    uint64_t *faces = new (std::nothrow) uint64_t[2 * F];
    uint64_t *cell_faces = new (std::nothrow) uint64_t[6 * N];
    uint64_t *nbrs = new (std::nothrow) uint64_t[6 * N];
    double *centers = new (std::nothrow) double[3 * N];
    uint64_t *face_index = new (std::nothrow) uint64_t[6 * N];
    if (!points || !cells || !faces || !cell_faces || !nbrs || !centers || !face_index) {
        delete[] points; delete[] cells; delete[] faces; delete[] cell_faces; delete[] nbrs; delete[] centers;
        delete[] face_index;
        return MC_ERR_NOMEM;
    }
    for (uint64_t i = 0; i < P; i++) {
        const uint64_t x = i % px, y = (i / px) % py, z = i / (px * py);
        points[3 * i] = (double)x * dx;
        points[3 * i + 1] = (double)y * dy;
        points[3 * i + 2] = (double)z * dz;
    }
    const uint64_t B = UINT64_MAX;
    for (uint64_t z = 0; z < ez; z++)
        for (uint64_t y = 0; y < ey; y++)
            for (uint64_t x = 0; x < ex; x++) {
                const uint64_t c = z * ex * ey + y * ex + x;
                const uint64_t g = x + y * px + z * px * py;
                uint64_t *n = cells + 8 * c;
                n[0] = g;
                n[1] = g + 1;
                n[2] = g + px;
                n[3] = g + px + 1;
                n[4] = g + px * py;
                n[5] = g + px * py + 1;
                n[6] = g + px * py + px;
                n[7] = g + px * py + px + 1;
                uint64_t *nb = nbrs + 6 * c;
                nb[0] = (z == 0) ? B : c - ex * ey;
                nb[1] = (z == ez - 1) ? B : c + ex * ey;
                nb[2] = (x == 0) ? B : c - 1;
                nb[3] = (x == ex - 1) ? B : c + 1;
                nb[4] = (y == 0) ? B : c - ex;
                nb[5] = (y == ey - 1) ? B : c + ex;
            }
    for (uint64_t i = 0; i < 6 * N; i++) face_index[i] = UINT64_MAX;
    uint64_t count = 0;
    for (uint64_t c = 0; c < N; c++)
        for (uint64_t f = 0; f < 6; f++) {
            if (face_index[6 * c + f] == UINT64_MAX) {
                const uint64_t nb_block = nbrs[6 * c + f];
                const uint64_t nb = (nb_block == B) ? N + f : nb_block;
                faces[2 * count] = c < nb ? c : nb;
                faces[2 * count + 1] = c < nb ? nb : c;
                if (nb_block < N) face_index[6 * nb_block + (f ^ 1)] = count;
                cell_faces[6 * c + f] = count++;
            } else {
                cell_faces[6 * c + f] = face_index[6 * c + f];
            }
        }
    delete[] face_index;
    for (uint64_t c = 0; c < N; c++) {
        double sx = 0.0, sy = 0.0, sz = 0.0;
        for (int i = 0; i < 8; i++) {
            const uint64_t p = cells[8 * c + i];
            sx += points[3 * p];
            sy += points[3 * p + 1];
            sz += points[3 * p + 2];
        }
        centers[3 * c] = sx / 8.0;
        centers[3 * c + 1] = sy / 8.0;
        centers[3 * c + 2] = sz / 8.0;
    }
    out->cells = N;
    out->faces = F;
    out->points = P;
    out->points_xyz = points;
    out->cell_nodes = cells;
    out->face_cells = faces;
    out->cell_faces = cell_faces;
    out->cell_neighbours = nbrs;
    out->cell_centers = centers;
    // FRONT, BACK, DOWN, UP walls; LEFT inlet; RIGHT outlet (mesh_examples.cpp:469-474)
    const uint64_t types[6] = {1, 1, 2, 3, 1, 1};
    for (int s = 0; s < 6; s++) out->boundary_types[s] = types[s];
    return count == F ? MC_OK : MC_ERR_MESH;
}

extern "C" void mc_mesh_box_destroy(mc_mesh_view *m)
{
    if (!m) return;
    delete[] m->points_xyz;
    delete[] m->cell_nodes;
    delete[] m->face_cells;
    delete[] m->cell_faces;
    delete[] m->cell_neighbours;
    delete[] m->cell_centers;
    memset(m, 0, sizeof(*m));
}

// Validate a mesh and return the reverse Cuthill-McKee cell order the
// solver uses with MC_REORDER_RCM (host only, no device work).
extern "C" int mc_mesh_rcm_order(const mc_mesh_view *mesh, int *cell_new_to_old)
{
    if (!mesh || !cell_new_to_old) return MC_ERR_ARG;
    mcb::HostMesh hm;
    std::string err;
    int rc;
    try {
        rc = mcb::build_host_mesh(mesh, mcb::HostPhysics{1.0}, hm, err);
        if (rc) return rc;
        std::vector<int> order;
        mcb::rcm_cell_order(hm, order);
        std::copy(order.begin(), order.end(), cell_new_to_old);
    } catch (const std::bad_alloc &) {
        return MC_ERR_NOMEM;
    }
    return MC_OK;
}
