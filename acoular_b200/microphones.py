"""Microphone array geometry, mirroring ``MicGeom`` (acoular/microphones.py:27-275).

Positions are a ``(3, num_mics)`` float64 array (rows x, y, z).  ``invalid_channels`` removes
columns as in acoular/microphones.py:174-179; XML import reads ``<pos Name x y z>`` elements as in
acoular/microphones.py:200-235.
"""

from __future__ import annotations

import hashlib
import xml.dom.minidom

import numpy as np


class MicGeom:
    def __init__(self, pos_total=None, file: str | None = None, invalid_channels=()):
        self.invalid_channels = list(invalid_channels)
        self.file = file
        if file is not None:
            doc = xml.dom.minidom.parse(file)
            xyz = [[float(el.getAttribute(a)) for a in 'xyz'] for el in doc.getElementsByTagName('pos')]
            self.pos_total = np.array(xyz, 'd').swapaxes(0, 1)
        elif pos_total is not None:
            self.pos_total = np.asarray(pos_total, dtype=np.float64).reshape(3, -1)
        else:
            self.pos_total = np.zeros((3, 0))

    @property
    def pos(self) -> np.ndarray:
        if len(self.invalid_channels) == 0:
            return self.pos_total
        keep = [i for i in range(self.pos_total.shape[-1]) if i not in self.invalid_channels]
        return self.pos_total[:, np.array(keep, dtype=int)]

    @property
    def num_mics(self) -> int:
        return self.pos.shape[-1]

    @property
    def center(self):
        if self.pos.any():
            c = np.average(self.pos, axis=1)
            c[abs(c) < 1e-16] = 0.0
            return c
        return None

    @property
    def digest(self) -> str:
        p = np.ascontiguousarray(self.pos)
        return '_' + hashlib.blake2b(p.tobytes() + str(p.shape).encode(), digest_size=16).hexdigest()


def disk_mics(num_mics: int, radius: float, seed: int, z: float = 0.0) -> MicGeom:
    """Seeded uniform layout in a planar disk: r = radius*sqrt(U), theta = 2*pi*U (``RandomState``)."""
    rng = np.random.RandomState(seed)
    r = radius * np.sqrt(rng.uniform(size=num_mics))
    th = 2 * np.pi * rng.uniform(size=num_mics)
    return MicGeom(pos_total=np.vstack([r * np.cos(th), r * np.sin(th), np.full(num_mics, z)]))


def log_spiral_mics(num_mics: int, diameter: float, seed: int, arms: int = 16) -> MicGeom:
    """Seeded multi-arm logarithmic spiral layout in the plane z = 0."""
    rng = np.random.RandomState(seed)
    per_arm = int(np.ceil(num_mics / arms))
    rmax = diameter / 2
    rmin = rmax * 0.05
    pts = []
    for a in range(arms):
        phase = 2 * np.pi * a / arms + rng.uniform(0, 0.05)
        for j in range(per_arm):
            t = (j + 0.5) / per_arm
            r = rmin * (rmax / rmin) ** t
            th = phase + 1.2 * np.pi * t
            pts.append((r * np.cos(th), r * np.sin(th), 0.0))
    p = np.array(pts[:num_mics]).T
    return MicGeom(pos_total=p)
