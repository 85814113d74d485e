"""Golden vectors of the headless surfacing functions, produced by the
reference's own code (oracle/_ref/ref_surface, built by oracle/build_ref_mesh.sh
from SphereUnionSurfacing.cpp, ForwardSimulation.cpp and Grid.cpp):

  * MarchingCubesPointCloud's fields (DiffMPMAnimator3D.cpp:488-514): P2G_Mass
    of the points on a coarse grid, G2G_Mass onto a grid refined by `quality`,
    and igl::marching_cubes of the fine masses at iso_mass;
  * SphereUnionMarchingCubesSurfaceFromPointCloud's mesh
    (SphereUnionSurfacing.cpp:7-128).

The point cloud is the reference's own point cloud of the torus test mesh
(mesh_torus_points.npz).  The GUI defaults (iso_mass 0.5, quality 4, sphere
radius 0.5, 2 blur passes for a unit grid; DiffMPMAnimator3D.cpp:735-743) are
scaled to this cloud's grid spacing; quality 2 keeps the fine grid small.

    bash oracle/build_ref_mesh.sh && python tests/golden/make_surface_golden.py
"""
from __future__ import annotations

import hashlib
import os
import subprocess
import sys
import tempfile

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(os.path.dirname(HERE))
REF = os.path.join(REPO, "oracle", "_ref", "ref_surface")

# the workload: the torus point cloud on a 0.05 grid over [-1, 1]^3
GRID_DX, QUALITY, ISO_MASS = 0.05, 2.0, 0.5
SPHERE_RADIUS, SPHERE_ISO, BLUR = 0.025, 0.025, 2
BOX_MIN, BOX_MAX = (-1.0, -1.0, -1.0), (1.0, 1.0, 1.0)


def main():
    sys.path.insert(0, REPO)
    from oracle import surface as osurf

    pts = np.load(os.path.join(HERE, "mesh_torus_points.npz"))["points"].astype(np.float32)
    with tempfile.TemporaryDirectory() as tmp:
        pf = os.path.join(tmp, "pts.f32")
        pts.tofile(pf)
        box = [repr(float(v)) for v in BOX_MIN + BOX_MAX]
        mass_out = os.path.join(tmp, "mass.bin")
        subprocess.check_call([REF, "mass", pf, "1.0", repr(GRID_DX), repr(QUALITY), repr(ISO_MASS), *box, mass_out])
        cd, cm, fd, fm, mv, mf = osurf.read_blocks(mass_out, "lflffi")
        sph_out = os.path.join(tmp, "sph.bin")
        sdx = GRID_DX / QUALITY
        subprocess.check_call([REF, "spheres", pf, repr(SPHERE_RADIUS), repr(float(np.float32(sdx))), repr(SPHERE_ISO),
                               str(BLUR), *box, sph_out])
        sv, sf = osurf.read_blocks(sph_out, "fi")
        # pin the oracle's sphere field: libigl's marching cubes of it must give the reference's mesh
        dims = osurf.grid_dims(BOX_MIN, BOX_MAX, np.float32(sdx))
        field = osurf.sphere_field(pts, SPHERE_RADIUS, np.float32(sdx), BLUR, BOX_MIN, dims)
        ff = os.path.join(tmp, "field.f32")
        field.astype(np.float32).tofile(ff)
        mc_out = os.path.join(tmp, "mc.bin")
        subprocess.check_call([REF, "mc", ff, str(dims[0]), repr(float(np.float32(sdx))), repr(SPHERE_ISO),
                               *box[:3], mc_out])
        ov, of = osurf.read_blocks(mc_out, "fi")
    print("mass grids", tuple(cd), tuple(fd), "mass mesh", len(mv) // 3, len(mf) // 3,
          "sphere mesh", len(sv) // 3, len(sf) // 3)
    pinned = np.array_equal(ov, sv) and np.array_equal(of, sf)
    print("oracle sphere field -> reference mesh:", pinned)
    if not pinned:
        raise SystemExit("the oracle's sphere field does not reproduce the reference's mesh")
    # the field itself (80^3 floats) is kept as a digest of its bytes
    sha = hashlib.sha256(field.astype(np.float32).tobytes()).hexdigest()
    np.savez_compressed(os.path.join(HERE, "surface_torus.npz"), grid_dx=np.float32(GRID_DX),
                        quality=np.float32(QUALITY), iso_mass=np.float32(ISO_MASS),
                        sphere_radius=np.float32(SPHERE_RADIUS), sphere_iso=np.float32(SPHERE_ISO),
                        blur=np.int32(BLUR), box_min=np.float32(BOX_MIN), box_max=np.float32(BOX_MAX),
                        coarse_dims=cd, coarse_mass=cm, fine_dims=fd, fine_mass=fm, mass_V=mv, mass_F=mf,
                        sphere_V=sv, sphere_F=sf, sphere_dims=np.int64(dims), sphere_dx=np.float32(sdx),
                        sphere_field_sha256=np.array(sha))


if __name__ == "__main__":
    main()
