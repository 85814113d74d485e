// stages_check.cpp -- the stage-level compat API (SingleThreadMPM::P_op_1, G_Reset,
// P2G, G_op, G2P, P_op_2 and MultiThreadMPM::ForwardTimeStep) used as a caller that
// composes its own time step would use the reference's: one step stage by stage must
// equal the engine's fused SingleThreadMPM::ForwardTimeStep (whose parity with the
// reference the other tests cover), and G_op's point-gravity form must follow the
// reference's formula (ForwardSimulation.cpp:200-224).  Prints the largest relative
// differences; exit status 1 when one exceeds its tolerance.
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <memory>
#include <vector>

#include "DiffMPMLib3D/ForwardSimulation.h"
#include "DiffMPMLib3D/MultiThreadForwardSimulation.h"

using namespace DiffMPMLib3D;

static uint64_t rng_state = 12345;
static float urand() {  // deterministic uniform [0, 1)
    rng_state = rng_state * 6364136223846793005ull + 1442695040888963407ull;
    return (float)((rng_state >> 40) & 0xFFFFFF) / 16777216.f;
}

static double rel_vec(const PointCloud& a, const PointCloud& b, int field) {
    double num = 0, den = 0;
    for (size_t p = 0; p < a.points.size(); p++) {
        const MaterialPoint& x = a.points[p];
        const MaterialPoint& y = b.points[p];
        const int w = field < 2 ? 3 : 9;
        for (int k = 0; k < w; k++) {
            float u = 0, v = 0;
            if (field == 0) { u = x.x[k]; v = y.x[k]; }
            if (field == 1) { u = x.v[k]; v = y.v[k]; }
            if (field == 2) { u = x.F.d[k]; v = y.F.d[k]; }
            if (field == 3) { u = x.C.d[k]; v = y.C.d[k]; }
            num = std::fmax(num, std::fabs((double)u - v));
            den = std::fmax(den, std::fabs((double)v));
        }
    }
    return den > 0 ? num / den : num;
}

int main() {
    const int n = 3000, dim = 16;
    const float dx = 1.f / dim, dt = 2e-4f, drag = 0.1f, s = 0.05f;
    const Vec3 f(0.f, -1.f, 0.f), mn(0.f, 0.f, 0.f);
    PointCloud cloud;
    cloud.points.resize(n);
    for (auto& mp : cloud.points) {
        mp.x = Vec3(0.3f + 0.4f * urand(), 0.3f + 0.4f * urand(), 0.3f + 0.4f * urand());
        mp.v = Vec3(0.2f * (urand() - 0.5f), 0.2f * (urand() - 0.5f), 0.2f * (urand() - 0.5f));
        mp.F = Mat3::Identity();
        for (int k = 0; k < 9; k++) {
            mp.F.d[k] += 0.05f * (urand() - 0.5f);
            mp.dFc.d[k] = 0.01f * (urand() - 0.5f);
        }
        mp.m = 1.5e-5f;
        mp.vol = 1.5e-5f;
        mp.lam = 1e3f;
        mp.mu = 7e2f;
    }
    // fused step
    PointCloud currA = cloud, nextA = cloud;
    Grid gA(dim, dim, dim, dx, mn);
    SingleThreadMPM::ForwardTimeStep(nextA, currA, gA, s, dt, drag, f);
    // the same step stage by stage
    PointCloud currB = cloud, nextB = cloud;
    Grid gB(dim, dim, dim, dx, mn);
    SingleThreadMPM::P_op_1(currB);
    SingleThreadMPM::G_Reset(gB);
    SingleThreadMPM::P2G(currB, gB, dt, drag);
    SingleThreadMPM::G_op(gB, dt, f);
    SingleThreadMPM::G2P(nextB, currB, gB);
    SingleThreadMPM::P_op_2(nextB, currB, s, dt);
    const double ex = rel_vec(nextB, nextA, 0), ev = rel_vec(nextB, nextA, 1), eF = rel_vec(nextB, nextA, 2),
                 eC = rel_vec(nextB, nextA, 3);
    // multi-threaded step = single-threaded step without smoothing
    PointCloud currC = cloud, nextC = cloud, currD = cloud, nextD = cloud;
    Grid gC(dim, dim, dim, dx, mn), gD(dim, dim, dim, dx, mn);
    std::vector<std::shared_ptr<Grid>> proxies;
    MultiThreadMPM::ForwardTimeStep(nextC, currC, gC, proxies, dt, drag, f);
    SingleThreadMPM::ForwardTimeStep(nextD, currD, gD, 0.f, dt, drag, f);
    const double emt = std::fmax(rel_vec(nextC, nextD, 0), rel_vec(nextC, nextD, 2));
    // point gravity: v = p / m + dt * mag * (g - x) / |g - x| where |m| > FLT_EPSILON
    Grid gG(4, 4, 4, 0.5f, Vec3(-1.f, -1.f, -1.f));
    int q = 0;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++, q++) {
                GridNode& nd = gG.nodes[i][j][k];
                nd.m = (q % 5 == 0) ? 0.f : 0.5f + 0.01f * q;
                nd.p = Vec3(0.1f * q, -0.05f * q, 0.02f);
                nd.v = Vec3(7.f, 7.f, 7.f);  // kept where the node is empty
            }
    const Vec3 gp(-0.5f, 0.f, 0.5f);  // a node position: zero force there
    SingleThreadMPM::G_op(gG, 0.1f, gp, 9.8f);
    double eg = 0;
    q = 0;
    for (int i = 0; i < 4; i++)
        for (int j = 0; j < 4; j++)
            for (int k = 0; k < 4; k++, q++) {
                const GridNode& nd = gG.nodes[i][j][k];
                const float xg[3] = {-1.f + 0.5f * i, -1.f + 0.5f * j, -1.f + 0.5f * k};
                float want[3];
                if (!(std::fabs(nd.m) > 1.1920929e-07f)) {
                    want[0] = want[1] = want[2] = 7.f;
                } else {
                    float d[3] = {gp[0] - xg[0], gp[1] - xg[1], gp[2] - xg[2]};
                    const float len = std::sqrt(d[0] * d[0] + d[1] * d[1] + d[2] * d[2]);
                    for (int a = 0; a < 3; a++) {
                        const float fa = len > 0.f ? d[a] / len * 9.8f : 0.f;
                        want[a] = nd.p[a] / nd.m + 0.1f * fa;
                    }
                }
                for (int a = 0; a < 3; a++) eg = std::fmax(eg, std::fabs((double)nd.v[a] - want[a]));
            }
    std::printf("stages x %.3g v %.3g F %.3g C %.3g  multithread %.3g  gravity %.3g\n", ex, ev, eF, eC, emt, eg);
    const bool ok = ex < 1e-6 && ev < 1e-4 && eF < 1e-5 && eC < 1e-3 && emt < 1e-5 && eg < 1e-5;
    return ok ? 0 : 1;
}
