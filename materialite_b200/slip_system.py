"""Slip systems (materialite/slip_system.py:17-173): unit plane normals and slip
directions, and the Schmid tensors d (x) n used by the crystal-plasticity update."""

import numpy as np

from .tensor import Vector


class SlipSystem:
    def __init__(self, normals, directions):
        self.normal = normals.unit
        self.direction = directions.unit

    def __len__(self):
        return len(self.normal)

    def __repr__(self):
        return ("SlipSystem(normals: " + str(np.round(self.normal.components, 3))
                + ",\n directions: " + str(np.round(self.direction.components, 3)) + ")")

    @classmethod
    def octahedral(cls):
        """The 12 FCC {111}<110> systems in the reference's order (slip_system.py:35-65)."""
        normals = [[1, 1, -1]] * 3 + [[1, -1, -1]] * 3 + [[1, -1, 1]] * 3 + [[1, 1, 1]] * 3
        directions = [[0, 1, 1], [1, 0, 1], [1, -1, 0], [0, 1, -1], [1, 0, 1], [1, 1, 0],
                      [0, 1, 1], [1, 0, -1], [1, 1, 0], [0, 1, -1], [1, 0, -1], [1, -1, 0]]
        return cls(Vector(normals, "s"), Vector(directions, "s"))

    @property
    def schmid_tensor(self):
        """d (x) n per system (slip_system.py:139-141)."""
        return self.direction.outer(self.normal)

    def schmid_mandel(self):
        """Mandel components of sym(d (x) n), shape (S, 6)."""
        return self.schmid_tensor.sym.components.reshape(-1, 6)
