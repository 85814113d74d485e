// Host-side parts of the compat C++ API called the way reference callers call
// them (no GPU needed): PointCloud's minibatch variants and
// Grid::QueryPoint_CubicBSpline / flatten / unflatten.
//   compat_host_check <in.bin> <out.bin>
// in:  int32 n, int32 nidx, int32 t0; float dLdF[9n], dFc[9n] (column-major);
//      int32 idx[nidx]; float lr, b1, b2, eps; then grid: int32 dims[3],
//      float dx, float min[3], int32 npts, float pts[3 npts]
// out: float norm, float dFc after two stochastic Adam steps (t0, t0 + 1) [9n],
//      then per query point: int32 count, count x int32 (i, j, k); then
//      int32 minibatch size and 1 if its indices are distinct and in range;
//      int32 1 if flatten / unflatten round-trips node masses
#include <cstdint>
#include <cstdio>
#include <fstream>
#include <set>
#include <vector>

#include "DiffMPMLib3D/Grid.h"
#include "DiffMPMLib3D/PointCloud.h"

using namespace DiffMPMLib3D;

template <class T> static T rd(std::ifstream& f) {
    T v;
    f.read(reinterpret_cast<char*>(&v), sizeof(T));
    return v;
}
template <class T> static void wr(std::ofstream& f, T v) { f.write(reinterpret_cast<const char*>(&v), sizeof(T)); }

int main(int argc, char** argv) {
    if (argc < 3) return 2;
    std::ifstream in(argv[1], std::ios::binary);
    const int n = rd<int32_t>(in), nidx = rd<int32_t>(in), t0 = rd<int32_t>(in);
    PointCloud pc;
    pc.points.resize((size_t)n);
    for (auto& p : pc.points)
        for (int k = 0; k < 9; k++) p.dLdF.data()[k] = rd<float>(in);
    for (auto& p : pc.points)
        for (int k = 0; k < 9; k++) p.dFc.data()[k] = rd<float>(in);
    std::vector<int> idx((size_t)nidx);
    for (int& i : idx) i = rd<int32_t>(in);
    const float lr = rd<float>(in), b1 = rd<float>(in), b2 = rd<float>(in), eps = rd<float>(in);
    int dims[3];
    for (int& d : dims) d = rd<int32_t>(in);
    const float dx = rd<float>(in);
    Vec3 mn;
    for (int a = 0; a < 3; a++) mn[a] = rd<float>(in);
    const int npts = rd<int32_t>(in);
    std::vector<Vec3> pts((size_t)npts);
    for (auto& q : pts)
        for (int a = 0; a < 3; a++) q[a] = rd<float>(in);

    std::ofstream out(argv[2], std::ios::binary);
    const float norm = pc.Compute_dLdF_Norm_Stochastic(idx);
    wr<float>(out, norm);
    pc.Descend_Adam_Stochastic(lr, norm, b1, b2, eps, t0, idx);
    pc.Descend_Adam_Stochastic(lr, norm, b1, b2, eps, t0 + 1, idx);
    for (auto& p : pc.points)
        for (int k = 0; k < 9; k++) wr<float>(out, p.dFc.data()[k]);

    Grid grid(dims[0], dims[1], dims[2], dx, mn);
    for (const Vec3& q : pts) {
        std::vector<std::array<int, 3>> ijk;
        const auto nodes = grid.QueryPoint_CubicBSpline(q, &ijk);
        wr<int32_t>(out, (int32_t)ijk.size());
        for (size_t e = 0; e < ijk.size(); e++) {
            for (int a = 0; a < 3; a++) wr<int32_t>(out, ijk[e][a]);
            // the returned references are the grid's own nodes
            if (&nodes[e].get() != &grid.nodes[ijk[e][0]][ijk[e][1]][ijk[e][2]]) return 3;
        }
        const Grid& cg = grid;
        if (cg.QueryPointConst_CubicBSpline(q).size() != nodes.size()) return 4;
    }
    const std::vector<int> mb = pc.generateMinibatchIndices(n, n / 3);
    const std::set<int> uniq(mb.begin(), mb.end());
    bool ok = uniq.size() == mb.size();
    for (int i : mb) ok &= i >= 0 && i < n;
    wr<int32_t>(out, (int32_t)mb.size());
    wr<int32_t>(out, ok ? 1 : 0);
    for (int i = 0; i < dims[0]; i++)
        for (int j = 0; j < dims[1]; j++)
            for (int k = 0; k < dims[2]; k++) grid.nodes[i][j][k].m = (float)((i * dims[1] + j) * dims[2] + k);
    Grid copy = grid;
    copy.unflatten(grid.flatten());
    bool round = true;
    for (int i = 0; i < dims[0]; i++)
        for (int j = 0; j < dims[1]; j++)
            for (int k = 0; k < dims[2]; k++) round &= copy.nodes[i][j][k].m == grid.nodes[i][j][k].m;
    wr<int32_t>(out, round ? 1 : 0);
    return 0;
}
