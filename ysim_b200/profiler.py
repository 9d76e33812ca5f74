"""Per-frame profile in the reference's FrameProfiler CSV schema.

profiler::FrameProfiler / FrameProfilerHistory (include/FrameProfiler.hpp):
each frame records its sequence number, wall time, frame milliseconds, fps
(1000 / frame_ms), the broad and narrow collision counts summed over its
substeps, and named section times summed over the frame.  The CSV has the
header ``frame_sequence,wall_time_seconds,frame_ms,fps,broad_collisions,
narrow_collisions`` followed by the section names (characters other than
letters, digits and '_' replaced by '_'), one row per kept frame (the last
``max_frames``), numbers as a C++ stream prints them (six significant digits).
"""
from __future__ import annotations

import collections
import dataclasses
import os
from typing import Dict, List


@dataclasses.dataclass
class FrameSnapshot:
    sequence: int = 0
    wall_time_seconds: float = 0.0
    frame_ms: float = 0.0
    fps: float = 0.0
    section_ms: List[float] = dataclasses.field(default_factory=list)
    broad_collisions: int = 0
    narrow_collisions: int = 0


def _num(v: float) -> str:
    """std::ostream << double with the default precision (6, %g)."""
    return "%g" % v


def _sanitize(name: str) -> str:
    return "".join(c if (c.isascii() and c.isalnum()) or c == "_" else "_" for c in name)


class FrameProfiler:
    def __init__(self, max_frames: int = 240):
        self.max_frames = max_frames
        self.section_names: List[str] = []
        self._lookup: Dict[str, int] = {}
        self.frames = collections.deque()
        self._open = False

    def ensure_section(self, name: str) -> int:
        if name not in self._lookup:
            self._lookup[name] = len(self.section_names)
            self.section_names.append(name)
        return self._lookup[name]

    def begin_frame(self, sequence: int, wall_time_seconds: float):
        self._cur = FrameSnapshot(sequence, wall_time_seconds, section_ms=[0.0] * len(self.section_names))
        self._open = True

    def add_collision_counts(self, broad: int, narrow: int):
        if self._open:
            self._cur.broad_collisions += int(broad)
            self._cur.narrow_collisions += int(narrow)

    def add_sample(self, name: str, ms: float):
        if not self._open:
            return
        i = self.ensure_section(name)
        if len(self._cur.section_ms) <= i:
            self._cur.section_ms += [0.0] * (i + 1 - len(self._cur.section_ms))
        self._cur.section_ms[i] += ms

    def end_frame(self, frame_ms: float):
        if not self._open:
            return
        s = self._cur
        s.frame_ms = frame_ms
        s.fps = 1000.0 / frame_ms if frame_ms > 0.0 else 0.0
        self.push(s)
        self._open = False

    def push(self, s: FrameSnapshot):
        if len(s.section_ms) < len(self.section_names):
            s.section_ms = s.section_ms + [0.0] * (len(self.section_names) - len(s.section_ms))
        self.frames.append(s)
        while len(self.frames) > self.max_frames:
            self.frames.popleft()

    def csv(self) -> str:
        lines = ["frame_sequence,wall_time_seconds,frame_ms,fps,broad_collisions,narrow_collisions"
                 + "".join("," + _sanitize(n) for n in self.section_names)]
        for f in self.frames:
            row = [str(f.sequence), _num(f.wall_time_seconds), _num(f.frame_ms), _num(f.fps),
                   str(f.broad_collisions), str(f.narrow_collisions)]
            row += [_num(f.section_ms[i] if i < len(f.section_ms) else 0.0) for i in range(len(self.section_names))]
            lines.append(",".join(row))
        return "\n".join(lines) + "\n"

    def export_csv(self, path: str) -> bool:
        d = os.path.dirname(path)
        if d:
            os.makedirs(d, exist_ok=True)
        try:
            with open(path, "w") as f:
                f.write(self.csv())
        except OSError:
            return False
        return True
