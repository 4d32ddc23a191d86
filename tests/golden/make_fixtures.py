"""Write the reference's own test data as fixtures (run where the reference tree exists).

The reference's image-model tests use the real-space potential
tests/data/3j9g_potential_ps4_4.mrc (a 64^3 float32 map, 4.4 A voxels;
cryojax tests/test_image_model.py:18-47, fixtures in tests/conftest.py).
mrcfile is not installed here, so this reads the MRC2014 layout directly:
a 1024-byte header (nx, ny, nz at bytes 0-11, mode at 12 (2 = float32),
cell lengths in A at 40-51, extended-header size nsymbt at 92), then the
data with x fastest, which is the [z][y][x] array mrcfile returns.

Output: tests/golden/3j9g_potential_ps4_4.npy and
tests/golden/3j9g_potential_ps4_4.json (voxel size, source).  Given the
reference's tests/data directory instead of the MRC path, it also copies
the RELION fixtures byte for byte into tests/golden/relion/: the STAR file
test_starfile.star (3 particles, one optics group) and the 3-image 16 x 16
stack 000000.mrcs it names (cryojax tests/test_relion_dataset.py:47-62).

    python tests/golden/make_fixtures.py /root/reference/tests/data
"""

import json
import os
import shutil
import struct
import sys

import numpy as np


def read_mrc(path):
    with open(path, "rb") as f:
        header = f.read(1024)
        nx, ny, nz, mode = struct.unpack("<4i", header[0:16])
        cx, cy, cz = struct.unpack("<3f", header[40:52])
        (nsymbt,) = struct.unpack("<i", header[92:96])
        if mode != 2:
            raise ValueError(f"expected float32 data (mode 2), got mode {mode}")
        f.seek(1024 + nsymbt)
        data = np.frombuffer(f.read(4 * nx * ny * nz), dtype="<f4").reshape(nz, ny, nx).copy()
    return data, float(cx / nx)


def main(src):
    here = os.path.dirname(os.path.abspath(__file__))
    if os.path.isdir(src):
        os.makedirs(os.path.join(here, "relion"), exist_ok=True)
        for name in ("test_starfile.star", "000000.mrcs"):
            shutil.copyfile(os.path.join(src, name), os.path.join(here, "relion", name))
        src = os.path.join(src, "3j9g_potential_ps4_4.mrc")
    vol, voxel = read_mrc(src)
    np.save(os.path.join(here, "3j9g_potential_ps4_4.npy"), vol)
    with open(os.path.join(here, "3j9g_potential_ps4_4.json"), "w") as f:
        json.dump({"voxel_size_A": voxel, "shape": list(vol.shape),
                   "source": "cryojax tests/data/3j9g_potential_ps4_4.mrc (MRC2014, mode 2)"}, f, indent=1)


if __name__ == "__main__":
    main(sys.argv[1])
