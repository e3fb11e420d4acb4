"""Checkpoint dumps of the tracking loop.

StepDumpBunch writes the reference's restart file format
(src/FFAG_dump.py:302-420): time-triggered, one ``time_{t_ns:.2f}_rank_{r}.npz``
per dump time with key ``particles`` = p-format N x 16 matrix of the
(optionally surviving) particles plus the dump time as column 17, appended
to an existing file (append_to_npz, src/FFAG_dump.py:1428-1448).  The file
is what main_track reads back with ``-r`` (examples/main_track.py:92-111).
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


class Dumps:
    """Registry of dump instances (src/FFAG_dump.py:1255-1284)."""

    def __init__(self):
        self.dumps = []

    def add_dump(self, dump_obj):
        self.dumps.append(dump_obj)

    def step_dumps(self):
        return [d for d in self.dumps if isinstance(d, StepDumpBunch)]

    def check_and_dump(self, time_Pre, time_Post, bunch_obj, data_type="RK4"):
        for d in self.dumps:
            d.check_and_dump(time_Pre, time_Post, bunch_obj, data_type)

    def list_dumps(self):
        for i, d in enumerate(self.dumps):
            print(f"Dump {i + 1}: {d.__class__.__name__}")
