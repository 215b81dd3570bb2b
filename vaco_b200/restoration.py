"""Host-side mirror of vaco's restoration geometry (src/restoration.rs:95-133).

`PlaneConfig.unit_counts()` and `unit_index()` follow vaco exactly; the CUDA
kernel tiles planes so that each tile lies in one unit of this mapping.
"""
from __future__ import annotations

from dataclasses import dataclass


@dataclass(frozen=True)
class PlaneConfig:
    width: int
    height: int
    bit_depth: int
    unit_size: int
    subsampling_y: bool

    def unit_counts(self):
        """Unit columns and rows, merging tails shorter than half a unit (:111-120)."""
        def count(extent):
            if self.unit_size == 0:
                return 1
            return max((extent + self.unit_size // 2) // self.unit_size, 1)
        return count(self.width), count(self.height)

    def unit_index(self, x: int, y: int) -> int:
        """Row-major unit index; vertical boundaries move up 8 luma rows (:124-133)."""
        cols, rows = self.unit_counts()
        row = min((y + (8 >> int(self.subsampling_y))) // self.unit_size, rows - 1)
        col = min(x // self.unit_size, cols - 1)
        return row * cols + col
