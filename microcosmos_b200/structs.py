"""State containers with the reference's field names and layouts
(src/microcosmos/structs/nodes.py:11-15, edges.py:15-21, fields.py:11-16).

Arrays are torch tensors on the device (float32 / int32); numpy arrays are accepted
on input and moved to the device by ``simulate``/``step``.
"""
from __future__ import annotations

import dataclasses
from typing import Any


@dataclasses.dataclass
class Nodes:
    position: Any      # (N, 2) (x, y)
    velocity: Any      # (N, 2)
    color_bend: Any    # (N,)   rendering only, carried through
    debug_vector: Any  # (N, 2) reset to zero every step by the PBD scheme

    def __replace__(self, **kw):
        return dataclasses.replace(self, **kw)

    def __len__(self):
        return len(self.position)


@dataclasses.dataclass
class Edges:
    pairs: Any                # (E, 2) int32 (src, tgt)
    theta: Any                # (E,)
    rest_lengths: Any         # (E,)
    bending_pairs: Any        # (B, 2) int32 (edge_in, edge_out)
    bending_rest_angles: Any  # (B,)
    bending_stiffness: Any    # (B,)

    def __replace__(self, **kw):
        return dataclasses.replace(self, **kw)


@dataclasses.dataclass
class Fields:
    grid_shape: tuple      # (H, W)
    steric: Any            # (H, W)
    fluid_velocity: Any    # (2, H, W)
    f_grid: Any            # (9, H, W) or None in recorded timeseries
    energy: Any = None

    def __replace__(self, **kw):
        return dataclasses.replace(self, **kw)
