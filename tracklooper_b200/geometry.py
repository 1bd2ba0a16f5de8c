"""LST geometry / module-map inputs (the event setup, "ES").

The reference reads these files from ``$LST_BASE/data/OT800_IT615_pt0.8``
(SDL/LSTESData.cc:14-75).  They ship packed as ``data/OT800_IT615_pt0.8.tar.xz``
and are unpacked next to it on first use, so that
``ES_BASE = <package dir>`` plays the role of ``$LST_BASE``.

On-disk formats (all little-endian, records back to back, no header):

* ``sensor_centroids.bin``: {u32 detId, f32 x, f32 y, f32 z, i32 type} with
  type 23 = PS pixel, 24 = PS strip, 25 = 2S (SDL/ModuleMethods.h:191-227).
* ``endcap_orientation.bin``: {u32 detId, f32 dxdy_slope, f32 centroid_phi}
  (SDL/EndcapGeometry.cc:13-41).
* ``tilted_barrel_orientation.bin``: {u32 detId, f32 drdz, f32 dxdy}
  (SDL/TiltedGeometry.cc:5-33).
* ``module_connection_tracing_merged.bin`` and ``pixelmap/pLS_map*.bin``:
  {u32 key, u32 n, n x u32 detId} (SDL/ModuleConnectionMap.cc:9-50).  For the
  pixel maps the key is a pLS superbin (0..44999); the charge-inclusive maps
  store it offset by 45000 (SDL/ModuleMethods.h:53).
"""
from __future__ import annotations

import lzma
import os
import tarfile
import threading

PKG_DIR = os.path.dirname(os.path.abspath(__file__))
DATA_DIR = os.path.join(PKG_DIR, "data")
GEOMETRY_NAME = "OT800_IT615_pt0.8"
ES_BASE = PKG_DIR  # plays the role of $LST_BASE: <ES_BASE>/data/<GEOMETRY_NAME>/...

_lock = threading.Lock()


# The geometries shipped (data/<name>.tar.xz): the pt0.8 module and pixel maps
# the reference loads (SDL/LSTESData.cc:46-57), and the pt0.6 ones beside them
# in the reference's data/, which it hard-codes away.  The event setup takes
# the pt cut of its cuts from the directory name (lst_es_info.ptCut).
GEOMETRIES = ("OT800_IT615_pt0.8", "OT800_IT615_pt0.6")


def geometry_dir(name: str = GEOMETRY_NAME) -> str:
    """Returns the unpacked geometry directory `name`, unpacking its tarball if needed."""
    out = os.path.join(DATA_DIR, name)
    marker = os.path.join(out, "sensor_centroids.bin")
    with _lock:
        if not os.path.exists(marker):
            tarball = os.path.join(DATA_DIR, name + ".tar.xz")
            if not os.path.exists(tarball):
                raise FileNotFoundError(f"geometry tarball missing: {tarball}")
            with lzma.open(tarball) as xz, tarfile.open(fileobj=xz) as tar:
                tar.extractall(DATA_DIR, filter="data")
    return out
