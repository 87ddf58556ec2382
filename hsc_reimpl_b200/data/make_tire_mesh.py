"""Extract the vehicle workload's tire mesh and tire placements from a checkout
of the reference into ``tire_tet4.npz`` beside this script.

    python -m hsc_reimpl_b200.data.make_tire_mesh [REFERENCE_ROOT]

Sources (paths inside the reference project):
  reproduction/vehicle_research/prepared/tire_tet4.npz      -- the Tet4 tire
      (3,548 nodes, 11,171 tets; BC_CONN: the 39 rim-connection nodes)
  reproduction/vehicle_research/prepared/scene_manifest.json -- where the
      tires sit: four mounted tires (E = 1e10) and the loose ones lying flat

The vehicle-scale system uses the four mounted tires and the first three loose
ones (seven tori, 24,836 nodes, 78,197 tets).  The mesh arrays are copied
unchanged (int32 / float64); nothing else of the reference is read.
"""
import json
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
OUT = HERE / "tire_tet4.npz"
MESH = "reproduction/vehicle_research/prepared/tire_tet4.npz"
SCENE = "reproduction/vehicle_research/prepared/scene_manifest.json"


def main(root="/root/reference"):
    root = Path(root)
    m = np.load(root / MESH)
    scene = json.loads((root / SCENE).read_text())
    tires = [i for i in scene["instances"] if i.get("geometry") == "tire_tet4.npz"]
    mounted = [i for i in tires if i["name"].startswith("mounted")]
    loose = [i for i in tires if i["name"].startswith("loose")][:3]
    used = mounted + loose
    np.savez_compressed(
        OUT,
        vertices=np.asarray(m["vertices"], dtype=np.float64),
        tetrahedra=np.asarray(m["tetrahedra"], dtype=np.int32),
        surface_triangles=np.asarray(m["surface_triangles"], dtype=np.int32),
        bc_conn=np.asarray(m["BC_CONN"], dtype=np.int32),
        bc_int=np.asarray(m["BC_INT"], dtype=np.int32),
        placement_translation=np.asarray([i["translation_m"] for i in used], dtype=np.float64),
        placement_rotation=np.asarray([i["rotation_matrix"] for i in used], dtype=np.float64),
        placement_mounted=np.asarray([i["name"].startswith("mounted") for i in used], dtype=np.int8),
        placement_name=np.asarray([i["name"] for i in used]),
    )
    print(f"wrote {OUT}: {m['vertices'].shape[0]} nodes, {m['tetrahedra'].shape[0]} tets, "
          f"{len(used)} placements")


if __name__ == "__main__":
    main(*sys.argv[1:])
