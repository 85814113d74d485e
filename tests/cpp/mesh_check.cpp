// mesh_check.cpp -- the compat GeometryLoading API used the way the
// reference's LoadMPMPointCloudFromObj uses it (MPMPolyscope.cpp:27-40): read
// an OBJ, take its vertices' bounding box, sample the lattice points inside.
// Usage: mesh_check <mesh.obj> <point_dx> <out.bin>; writes the points as
// float32 triples.
#include <cfloat>
#include <cmath>
#include <cstdio>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "DiffMPMLib3D/GeometryLoading.h"

using namespace DiffMPMLib3D;

int main(int argc, char** argv) {
    if (argc != 4) return 2;
    std::ifstream in(argv[1]);
    std::vector<float> V;
    std::vector<int> F;
    std::string line;
    while (std::getline(in, line)) {
        std::istringstream ss(line);
        std::string tag;
        ss >> tag;
        if (tag == "v") {
            float x, y, z;
            ss >> x >> y >> z;
            V.insert(V.end(), {x, y, z});
        } else if (tag == "f") {
            std::string a, b, c;
            ss >> a >> b >> c;
            for (const std::string& t : {a, b, c}) F.push_back(std::stoi(t.substr(0, t.find('/'))) - 1);
        }
    }
    Vec3 mn(FLT_MAX, FLT_MAX, FLT_MAX), mx(-FLT_MAX, -FLT_MAX, -FLT_MAX);
    for (size_t i = 0; i < V.size() / 3; i++)
        for (int j = 0; j < 3; j++) {
            mn[j] = std::fmin(mn[j], V[3 * i + j]);
            mx[j] = std::fmax(mx[j], V[3 * i + j]);
        }
    std::vector<Vec3> pts = GeometryLoading::GeneratePointCloudFromWatertightTriangleMesh(
        GeometryLoading::TriMatrix<float>{&V}, GeometryLoading::TriMatrix<int>{&F}, mn, mx, std::stof(argv[2]));
    FILE* f = std::fopen(argv[3], "wb");
    if (!f) return 3;
    for (const Vec3& p : pts) std::fwrite(p.data(), sizeof(float), 3, f);
    std::fclose(f);
    std::printf("%zu\n", pts.size());
    return 0;
}
