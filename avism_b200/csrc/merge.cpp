// merge.cpp -- MERGE_VOID (src/voidfinding.f90:718-999) at the level of cubes.
//
// The reference walks the cubes in volume order and paints their cells into
// MARCA first-writer-wins.  The only cell-level questions it asks are
//   (a) for a cube that no earlier cube absorbed: the painted cell of its
//       1-cell halo box closest to its centre (ties: first in K,J,I order), and
//       the void id painted there;
//   (b) nothing else -- absorption uses a ball search on cube centres and an
//       integer box-overlap test.
// (a) is answered from the painted boxes themselves: the closest cell of a
// box to a point is the per-axis clamp, and the value painted on a cell is the
// owner of the earliest-painted box containing it.  Every cube that can touch
// cube i -- through (a) or through absorption, which needs overlapping 1-cell
// halo boxes -- is on i's neighbour list, built once on the GPU with the exact
// ball-search distance.  The merge therefore runs on cube records only
// (O(cubes x neighbours)); the cell grid is painted afterwards on the GPU from
// the recorded paint order.
#include <algorithm>
#include <climits>
#include <cmath>
#include <cstring>
#include <vector>

#include "merge.h"

namespace avism {

namespace {

// squared distance as distance() in src/kdtree.f90:1441-1465
[[maybe_unused]] inline float dist2_ref(float px, float py, float pz, float qx, float qy, float qz, float L, int periodic) {
    float dx = px - qx, dy = py - qy, dz = pz - qz;
    if (periodic) {
        float a = std::fabs(dx); dx = std::fmin(a, L - a);
        a = std::fabs(dy); dy = std::fmin(a, L - a);
        a = std::fabs(dz); dz = std::fmin(a, L - a);
    }
    float d = dx * dx;
    d = d + dy * dy;
    d = d + dz * dz;
    return d;
}

}  // namespace

float merge_ball_r2(float vol, float dx) {
    const float rthis = (std::sqrt(3.0f) / 2.0f) * std::pow(vol, 1.0f / 3.0f);
    const float rr = 2.0f * rthis + ((2.1f * std::sqrt(3.0f)) * dx) * 1.0f;
    return rr * rr;
}

void merge_cubes_host(const MergeIn &in, MergeOut &out) {
    const int32_t nv = in.nvoid;
    const int low1 = in.low1, low2 = in.low2;
    const float dx = in.dx;
    const int32_t *X0 = in.x0, *X1 = in.x1, *Y0 = in.y0, *Y1 = in.y1, *Z0 = in.z0, *Z1 = in.z1;
    const int32_t *father = in.father;
    out.uvoid.assign(nv, -1);
    out.gxc.resize(nv); out.gyc.resize(nv); out.gzc.resize(nv); out.volnew.resize(nv);
    out.paint_time.assign(nv, -1);
    out.paint_owner.assign(nv, 0);
    std::vector<float> &gxc = out.gxc, &gyc = out.gyc, &gzc = out.gzc, &vol = out.volnew;
    for (int32_t i = 0; i < nv; i++) {
        gxc[i] = in.rx1 + (float)(in.icx[i] - 1) * dx;
        gyc[i] = in.rx1 + (float)(in.icy[i] - 1) * dx;
        gzc[i] = in.rx1 + (float)(in.icz[i] - 1) * dx;
        vol[i] = ((in.rfx[i] - in.rix[i]) * (in.rfy[i] - in.riy[i])) * (in.rfz[i] - in.riz[i]);
    }
    std::vector<char> major(nv, 0);
    int32_t ptime = 0;
    int32_t nvoid2 = nv;
    auto paint = [&](int32_t cube, int32_t owner) {   // 1-based ids; each cube paints once
        const int c = cube - 1;
        if (out.paint_time[c] >= 0) return;
        out.paint_time[c] = ptime++;
        out.paint_owner[c] = owner;
    };
    auto absorb = [&](int32_t i0, int32_t i1) {       // src/voidfinding.f90:867-872
        const float v0 = vol[i0 - 1], v1 = vol[i1 - 1];
        gxc[i0 - 1] = (gxc[i0 - 1] * v0 + gxc[i1 - 1] * v1) / (v0 + v1);
        gyc[i0 - 1] = (gyc[i0 - 1] * v0 + gyc[i1 - 1] * v1) / (v0 + v1);
        gzc[i0 - 1] = (gzc[i0 - 1] * v0 + gzc[i1 - 1] * v1) / (v0 + v1);
        vol[i0 - 1] = v0 + v1;
    };
    std::vector<std::pair<float, int32_t>> ball;
    const long long ne = low2 - low1 + 1;
    for (int32_t I = 0; I < nv; I++) {
        const int32_t ind1 = in.indice[I];
        const int c1 = ind1 - 1;
        const int32_t *nb = in.nbr + in.nbr_start[c1];
        const int32_t nnb = in.nbr_start[c1 + 1] - in.nbr_start[c1];
        int32_t ind0, indp;
        if (out.uvoid[c1] > 0) {
            ind0 = out.uvoid[c1];
            indp = father[ind0 - 1];
        } else {
            ind0 = ind1;
            indp = father[ind0 - 1];
            // closest painted cell of the 1-cell halo box whose void has the same
            // father (src/voidfinding.f90:822-860); ties: first in K,J,I order.
            // Boxes of different fathers never overlap, so the painted boxes of
            // this cube's own neighbour list are all that can hold such a cell.
            const int e0[3] = {std::max(X0[c1] - 1, low1), std::max(Y0[c1] - 1, low1), std::max(Z0[c1] - 1, low1)};
            const int e1[3] = {std::min(X1[c1] + 1, low2), std::min(Y1[c1] + 1, low2), std::min(Z1[c1] + 1, low2)};
            const int cc[3] = {in.icx[c1], in.icy[c1], in.icz[c1]};
            long long bestkey = LLONG_MAX;
            int best[3] = {0, 0, 0};
            for (int32_t t = 0; t < nnb; t++) {
                const int32_t j = nb[t];
                if (out.paint_time[j] < 0) continue;
                const int lo[3] = {std::max(X0[j], e0[0]), std::max(Y0[j], e0[1]), std::max(Z0[j], e0[2])};
                const int hi[3] = {std::min(X1[j], e1[0]), std::min(Y1[j], e1[1]), std::min(Z1[j], e1[2])};
                if (lo[0] > hi[0] || lo[1] > hi[1] || lo[2] > hi[2]) continue;
                int q[3];
                long long d2 = 0;
                for (int a = 0; a < 3; a++) {
                    q[a] = std::min(std::max(cc[a], lo[a]), hi[a]);
                    d2 += (long long)(cc[a] - q[a]) * (cc[a] - q[a]);
                }
                const long long key = d2 * ne * ne * ne + ((long long)(q[2] - low1) * ne + (q[1] - low1)) * ne + (q[0] - low1);
                if (key < bestkey) { bestkey = key; best[0] = q[0]; best[1] = q[1]; best[2] = q[2]; }
            }
            if (bestkey != LLONG_MAX) {
                // value painted on that cell: owner of the earliest painted box holding it
                int32_t tmin = INT_MAX, own = 0;
                for (int32_t t = 0; t < nnb; t++) {
                    const int32_t j = nb[t];
                    const int32_t pt = out.paint_time[j];
                    if (pt < 0 || best[0] < X0[j] || best[0] > X1[j] || best[1] < Y0[j] || best[1] > Y1[j] ||
                        best[2] < Z0[j] || best[2] > Z1[j]) continue;
                    if (pt < tmin) { tmin = pt; own = out.paint_owner[j]; }
                }
                ind0 = own;
            }
            if (ind0 != ind1) {
                out.uvoid[c1] = ind0;
                absorb(ind0, ind1);
                paint(ind1, ind0);
                nvoid2--;
            } else {
                paint(ind0, ind0);
                major[ind0 - 1] = 1;
            }
        }
        // absorb the cubes of the ball search (src/voidfinding.f90:904-987) in
        // (distance, id) order; the overlap test on the 1-cell halo boxes is what
        // put them on the neighbour list
        ball.clear();
        for (int32_t t = 0; t < nnb; t++)
            if (in.nbr_inball[in.nbr_start[c1] + t]) ball.push_back({in.nbr_d2[in.nbr_start[c1] + t], nb[t]});
        std::sort(ball.begin(), ball.end());
        for (const auto &bj : ball) {
            const int32_t j = bj.second;
            const int32_t ind2 = j + 1;
            if (major[j]) continue;
            if (out.uvoid[j] >= 0) continue;
            if (indp != father[j]) continue;
            out.uvoid[j] = ind0;
            absorb(ind0, ind2);
            paint(ind2, ind0);
            nvoid2--;
        }
    }
    out.nvoid2 = nvoid2;
}

}  // namespace avism
