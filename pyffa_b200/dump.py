"""Checkpoint dumps of the tracking loop.

StepDumpBunch writes the reference's restart file format
(src/FFAG_dump.py:302-420): time-triggered, one ``time_{t_ns:.2f}_rank_{r}.npz``
per dump time with key ``particles`` = p-format N x 16 matrix of the
(optionally surviving) particles plus the dump time as column 17, appended
to an existing file (append_to_npz, src/FFAG_dump.py:1428-1448).  The file
is what main_track reads back with ``-r`` (examples/main_track.py:92-111).

PositionDumpBunch writes the azimuth-crossing file of the reference
(src/FFAG_dump.py:789-1130): every post-step row of a particle that crossed
the target azimuth in a step ending inside (start_time, end_time), saved once
the tracking time passes end_time as
``crossing_angle_{deg:.1f}_start_{t0_ns:.3f}_end_{t1_ns:.3f}_rank_{r}.npz``
(key ``particles``: p-format N x 16 rows with the RF phase reduced mod 2 pi,
plus the step's end time as column 17).  The crossing test itself runs in the
push kernels (ffa_push_crossing); this class holds the rows and writes them.
"""
from __future__ import annotations

import os
import sys

import numpy as np

from .constants import COLUMNS, FFAG_ConversionTools


def append_to_npz(filepath, new_data):
    if os.path.exists(filepath):
        combined = np.vstack((np.load(filepath)["particles"], new_data))
    else:
        combined = new_data
    np.savez_compressed(filepath, particles=combined)


class StepDumpBunch:
    def __init__(self, start_time, end_time, time_interval, filter_survive_flag=True, save_folder="dump_data",
                 rank=0, allow_existing=False):
        self.start_time = start_time
        self.end_time = end_time
        self.time_interval = time_interval
        self.save_folder = save_folder
        self.filter_survive_flag = filter_survive_flag
        self.rank = rank
        if rank == 0:
            if not os.path.exists(save_folder):
                os.makedirs(save_folder)
            elif os.listdir(save_folder) and not allow_existing:
                # the reference aborts every rank here (src/FFAG_dump.py:316-326)
                sys.stderr.write(f"Error: dump folder {save_folder} exists and is not empty\n")
                raise SystemExit(1)

    def check_and_dump(self, time_Pre, time_Post, bunch_obj, data_type):
        """The per-step trigger of the reference (src/FFAG_dump.py:330-356)."""
        if self.start_time < time_Post < self.end_time:
            a = (time_Pre - self.start_time) // self.time_interval
            b = (time_Post - self.start_time) // self.time_interval
            if a != b:
                self.dump_bunch(bunch_obj, time_Post, data_type)

    def dump_bunch(self, bunch_obj, time_Post, data_type):
        local = bunch_obj.LocalBunch
        surv = local[:, COLUMNS["Survive"]]
        parts = local[surv == 1, :] if self.filter_survive_flag else local
        if parts.shape[0] == 0:
            return
        conv = FFAG_ConversionTools()
        if data_type == "RK4":
            p = conv.ConvertVrzek2Przek(parts)
        elif data_type == "Boris":
            p = conv.ConvertVrzek2Przek_boris(parts)
        else:
            raise ValueError("data_type must be RK4 or Boris")
        fn = os.path.join(self.save_folder, f"time_{time_Post * 1e9:.2f}_rank_{self.rank}.npz")
        append_to_npz(fn, np.hstack((p, np.full((p.shape[0], 1), time_Post))))


class PositionDumpBunch:
    def __init__(self, target_azimuth_angle_deg, start_time, end_time, save_folder="dump_data", rank=0,
                 allow_existing=False):
        self.target_azimuth_angle = np.deg2rad(target_azimuth_angle_deg) % (2 * np.pi)
        self.save_folder = save_folder
        self.start_time = start_time
        self.end_time = end_time
        self.save_flag = False
        self.rank = rank
        self._rows = []
        self._records = []
        self.write_cursor = 0
        if rank == 0:
            if not os.path.exists(save_folder):
                os.makedirs(save_folder)
            elif os.listdir(save_folder) and not allow_existing:
                # the reference aborts every rank here (src/FFAG_dump.py:812-822)
                sys.stderr.write(f"Error: dump folder {save_folder} exists and is not empty\n")
                raise SystemExit(1)

    def in_window(self, t_post: np.ndarray) -> np.ndarray:
        """Steps whose crossings are recorded (src/FFAG_dump.py:1107)."""
        return (t_post < self.end_time) & (t_post > self.start_time)

    def add_particles(self, particle_data, time_i):
        """Appends v-format rows with the time column (src/FFAG_dump.py:965-993);
        time_i may be one value or one per row."""
        particle_data = np.asarray(particle_data, dtype=np.float64)
        t = np.broadcast_to(np.asarray(time_i, dtype=np.float64), (particle_data.shape[0],))
        self._rows.append(np.hstack((particle_data, t[:, None])))
        self.write_cursor += particle_data.shape[0]

    def add_records(self, records, t_post):
        """Keeps the raw crossing records behind the rows (layout of
        ffa_push_crossing, plus the step's end time as a last column): the
        pre-step state and the ratio let an analysis interpolate to the exact
        azimuth, which the saved post-step rows do not."""
        records = np.asarray(records, dtype=np.float64)
        t = np.broadcast_to(np.asarray(t_post, dtype=np.float64), (records.shape[0],))
        self._records.append(np.hstack((records, t[:, None])))

    @property
    def crossing_records(self) -> np.ndarray:
        if len(self._records) > 1:
            self._records = [np.vstack(self._records)]
        return self._records[0] if self._records else np.zeros((0, 24))

    @property
    def saved_data(self) -> np.ndarray:
        if len(self._rows) > 1:
            self._rows = [np.vstack(self._rows)]
        return self._rows[0] if self._rows else np.zeros((0, 17))

    def file_name(self) -> str:
        return (f"crossing_angle_{np.rad2deg(self.target_azimuth_angle):.1f}_start_{self.start_time * 1e9:.3f}"
                f"_end_{self.end_time * 1e9:.3f}_rank_{self.rank}.npz")

    def save_all_particles(self, data_type):
        """src/FFAG_dump.py:996-1026 (writes even when no particle crossed)."""
        data = self.saved_data
        conv = FFAG_ConversionTools()
        if data_type == "RK4":
            p = conv.ConvertVrzek2Przek(data[:, :-1])
        elif data_type == "Boris":
            p = conv.ConvertVrzek2Przek_boris(data[:, :-1])
        else:
            raise ValueError("data_type must be RK4 or Boris")
        p[:, 9] = np.mod(p[:, 9], 2 * np.pi)
        np.savez(os.path.join(self.save_folder, self.file_name()), particles=np.hstack((p, data[:, [-1]])))

    def check_and_dump(self, time_Pre, time_Post, bunch_obj, data_type):
        raise NotImplementedError("the azimuth-crossing test runs inside the push kernels; track with "
                                  "FFAG_RungeKutta's loops, which feed this dump")


def _prepare_folder(save_folder, rank, allow_existing):
    if rank == 0:
        if not os.path.exists(save_folder):
            os.makedirs(save_folder)
        elif os.listdir(save_folder) and not allow_existing:
            sys.stderr.write(f"Error: dump folder {save_folder} exists and is not empty\n")
            raise SystemExit(1)


class StepDump:
    """Time snapshots of selected particles, one file per particle
    (src/FFAG_dump.py:140-290): at every step whose [t_pre, t_post] crosses
    a new start_time + k * time_interval node (both inside the open window),
    the post-step rows of the tracked global IDs that were alive at the start
    of the step, converted to p-format, with t_post as column 17; written
    (``particle_{gid}_rank_{r}.npz``, key ``particles``) once t_pre passes
    end_time.  The tracking loop feeds it (record)."""

    def __init__(self, start_time, end_time, time_interval, tracked_particle_id_global, save_folder="dump_data",
                 rank=0, allow_existing=False):
        self.start_time, self.end_time = float(start_time), float(end_time)
        self.time_interval = float(time_interval)
        if not self.time_interval > 0:
            raise ValueError("time_interval must be > 0")
        self.save_folder = save_folder
        self.rank = rank
        self.tracked_global_ids = np.asarray(tracked_particle_id_global, dtype=np.int64)
        self.particle_buffer_dict = {}
        self.save_flag = False
        _prepare_folder(save_folder, rank, allow_existing)

    def fires(self, t_pre, t_post) -> np.ndarray:
        """The step trigger of check_and_dump (src/FFAG_dump.py:250-276)."""
        t_pre, t_post = np.asarray(t_pre), np.asarray(t_post)
        inside = (self.start_time < t_pre) & (t_pre < self.end_time) & (self.start_time < t_post) & \
            (t_post < self.end_time)
        eps = 1e-12
        a = np.floor((t_pre - self.start_time) / self.time_interval + eps)
        b = np.floor((t_post - self.start_time) / self.time_interval + eps)
        return inside & (a != b)

    def record(self, rows_v, alive_pre, time_stamp, data_type):
        """rows_v: post-step v-format rows of the tracked particles present in
        the bunch; alive_pre: their survival at the start of the step."""
        conv = FFAG_ConversionTools()
        for row, alive in zip(np.atleast_2d(rows_v), np.atleast_1d(alive_pre)):
            if not alive:
                continue
            st = row[None, :]
            c = conv.ConvertVrzek2Przek(st) if data_type == "RK4" else conv.ConvertVrzek2Przek_boris(st)
            gid = int(row[15])
            self.particle_buffer_dict.setdefault(gid, []).append(np.hstack((c.ravel(), [time_stamp])))

    def dump_all_particles(self):
        for gid, rows in self.particle_buffer_dict.items():
            if rows:
                np.savez_compressed(os.path.join(self.save_folder, f"particle_{gid}_rank_{self.rank}.npz"),
                                    particles=np.vstack(rows))

    def check_and_dump(self, time_Pre, time_Post, bunch_obj, data_type):
        raise NotImplementedError("StepDump is fed by FFAG_RungeKutta's loops")


class PositionDump:
    """Crossing records of selected particles, one file per particle
    (src/FFAG_dump.py:534-788): the post-step row of every tracked particle
    that crossed the target azimuth in a step ending inside (start_time,
    end_time), p-format with the RF phase reduced mod 2 pi and the step's end
    time as column 17, at most max_records per particle; written as
    ``particle_{gid}_angle_{deg:.1f}_rank_{r}.npz`` once the tracking time
    passes end_time.  The crossing test runs in the push kernels."""

    def __init__(self, target_azimuth_angle_deg, start_time, end_time, tracked_particle_id_global,
                 save_folder="dump_data", max_records=10000, rank=0, allow_existing=False):
        self.target_azimuth_angle = np.deg2rad(target_azimuth_angle_deg) % (2 * np.pi)
        self.start_time, self.end_time = start_time, end_time
        self.tracked_global_ids = np.asarray(tracked_particle_id_global, dtype=np.int64)
        self.save_folder = save_folder
        self.max_records = max_records
        self.save_flag = False
        self.rank = rank
        self.particle_buffer_dict = {}
        _prepare_folder(save_folder, rank, allow_existing)

    def in_window(self, t_post):
        return (t_post < self.end_time) & (t_post > self.start_time)

    def add_particles(self, rows_v, time_i, data_type="Boris"):
        rows_v = np.atleast_2d(rows_v)
        keep = np.isin(rows_v[:, 15].astype(np.int64), self.tracked_global_ids)
        if not keep.any():
            return
        rows_v = rows_v[keep]
        t = np.broadcast_to(np.asarray(time_i, dtype=np.float64), keep.shape)[keep]
        conv = FFAG_ConversionTools()
        c = conv.ConvertVrzek2Przek(rows_v) if data_type == "RK4" else conv.ConvertVrzek2Przek_boris(rows_v)
        c[:, 9] = np.mod(c[:, 9], 2 * np.pi)
        full = np.hstack((c, t[:, None]))
        for gid, row in zip(rows_v[:, 15].astype(np.int64), full):
            buf = self.particle_buffer_dict.setdefault(int(gid), [])
            if len(buf) < self.max_records:
                buf.append(row)

    def save_all_particles(self, data_type=None):
        deg = np.rad2deg(self.target_azimuth_angle)
        for gid, rows in self.particle_buffer_dict.items():
            if rows:
                np.savez(os.path.join(self.save_folder, f"particle_{gid}_angle_{deg:.1f}_rank_{self.rank}.npz"),
                         particles=np.vstack(rows))

    def check_and_dump(self, time_Pre, time_Post, bunch_obj, data_type):
        raise NotImplementedError("PositionDump is fed by FFAG_RungeKutta's loops")


class Dumps:
    """Registry of dump instances (src/FFAG_dump.py:1255-1284)."""

    def __init__(self):
        self.dumps = []

    def add_dump(self, dump_obj):
        self.dumps.append(dump_obj)

    def step_dumps(self):
        return [d for d in self.dumps if isinstance(d, StepDumpBunch)]

    def position_dumps(self):
        return [d for d in self.dumps if isinstance(d, (PositionDumpBunch, PositionDump))]

    def particle_step_dumps(self):
        return [d for d in self.dumps if isinstance(d, StepDump)]

    def check_and_dump(self, time_Pre, time_Post, bunch_obj, data_type="RK4"):
        for d in self.dumps:
            d.check_and_dump(time_Pre, time_Post, bunch_obj, data_type)

    def list_dumps(self):
        for i, d in enumerate(self.dumps):
            print(f"Dump {i + 1}: {d.__class__.__name__}")
