"""Fan-beam geometry record (no native library needed to import it).

Field meaning follows the reference's ``Projector`` members
(ReconNet4D/Projector.h:10-37) and ``Grid`` / ``Detector``
(ReconNet4D/Siddon.h:20-76).  Keeping it apart from the device API lets the
synthetic-input generators and the CPU-only reference arm of the benchmark
describe a workload without loading the sm_100a library.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass
class FanGeometry:
    """Fan-beam geometry; ``da`` is the angular detector pitch in radians
    (du_mm / dsd, python/ReconNet_no_tf.py:44)."""
    nx: int = 512
    ny: int = 512
    nz: int = 1
    dx: float = 1.0
    dy: float = 1.0
    dz: float = 1.0
    nu: int = 736
    nv: int = 1
    da: float = 1.2858 / 1085.6
    dv: float = 1.0
    off_a: float = 0.0
    off_v: float = 0.0
    dsd: float = 1085.6
    dso: float = 595.0
    cx: float = 0.0
    cy: float = 0.0
    cz: float = 0.0

    def native(self, nbatches: int, nchannels: int, nview: int):
        """The C-ABI ``RnFanGeom`` record of this geometry (loads the library)."""
        from . import _native as N
        g = N.RnFanGeom()
        g.nBatches, g.nChannels = int(nbatches), int(nchannels)
        g.nx, g.ny, g.nz = int(self.nx), int(self.ny), int(self.nz)
        g.dx, g.dy, g.dz = float(self.dx), float(self.dy), float(self.dz)
        g.cx, g.cy, g.cz = float(self.cx), float(self.cy), float(self.cz)
        g.nu, g.nview, g.nv = int(self.nu), int(nview), int(self.nv)
        g.du, g.dv = float(self.da), float(self.dv)
        g.off_u, g.off_v = float(self.off_a), float(self.off_v)
        g.dsd, g.dso = float(self.dsd), float(self.dso)
        return g


@dataclass
class CylGeometry:
    """Cylindrical-detector cone-beam geometry on a circular orbit (RnCylGeom):
    nx x ny x nz voxels of dx x dy x dz mm centred at (cx, cy, cz); nu x nv
    detector cells, ``da`` rad apart in fan angle and ``dv`` mm apart in
    height at the detector, offsets in cells; source-to-detector ``dsd`` and
    source-to-isocentre ``dso`` in mm.  Defaults: the 512 x 512 x 128 volume,
    736 x 64 cells and 1085.6 / 595 mm distances of the cone-beam workload."""
    nx: int = 512
    ny: int = 512
    nz: int = 128
    dx: float = 0.8
    dy: float = 0.8
    dz: float = 1.0
    cx: float = 0.0
    cy: float = 0.0
    cz: float = 0.0
    nu: int = 736
    nv: int = 64
    da: float = 1.2858 / 1085.6
    dv: float = 1.0
    off_a: float = 0.0
    off_v: float = 0.0
    dsd: float = 1085.6
    dso: float = 595.0

    def native(self, nbatches: int, nview: int):
        from . import _native as N
        g = N.RnCylGeom()
        g.nBatches = int(nbatches)
        g.nx, g.ny, g.nz = int(self.nx), int(self.ny), int(self.nz)
        g.dx, g.dy, g.dz = float(self.dx), float(self.dy), float(self.dz)
        g.cx, g.cy, g.cz = float(self.cx), float(self.cy), float(self.cz)
        g.nu, g.nview, g.nv = int(self.nu), int(nview), int(self.nv)
        g.da, g.dv = float(self.da), float(self.dv)
        g.off_a, g.off_v = float(self.off_a), float(self.off_v)
        g.dsd, g.dso = float(self.dsd), float(self.dso)
        return g
