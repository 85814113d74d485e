// Reads an .mpmbin with the compat PointCloud and writes it back (host IO only).
#include <cstdio>
#include "DiffMPMLib3D/PointCloud.h"
using namespace DiffMPMLib3D;
int main(int argc, char** argv) {
    if (argc != 3) return 2;
    PointCloud pc;
    if (!pc.ReadEntirePointCloudFromBinaryFile(argv[1])) return 1;
    pc.WriteEntirePointCloudToBinaryFile(argv[2]);
    std::printf("%zu\n", pc.points.size());
    return 0;
}
