"""The job client's event protocol (core/solve_worker.py:44-153), on the CPU:
status records written by hand are turned into the same events the
reference's client gives, the result is delivered once, a worker that exits
without a status is reported with its log, and cleanup removes the files."""

import json
import os
import pickle
import subprocess
import sys

import pytest

from voxelsim_fea_b200.solve_worker import SolverClient, _JobFiles


def _client_with_files():
    c = SolverClient()
    c._files = _JobFiles()
    return c


def _status(c, **rec):
    with open(c._files.status, "w") as fh:
        json.dump(rec, fh)


def test_phases_map_to_events():
    c = _client_with_files()
    try:
        assert c.poll() == ("running", 0.0)
        _status(c, phase="voxel", frac=0.25)
        assert c.poll() == ("voxel", 0.25)
        _status(c, phase="solve", frac=0.0)
        assert c.poll() == ("solve", None)
        _status(c, phase="solve", frac=0.0, cg_iter=7, cg_resid=1e-3, cg_tol=1e-6)
        assert c.poll() == ("solve", {"iter": 7, "resid": 1e-3, "tol": 1e-6})
        _status(c, phase="something-new")
        assert c.poll() == ("running", 0.0)
        _status(c, phase="done", frac=1.0)
        ev = c.poll()
        assert ev[0] == "error" and ev[1].startswith("could not read solver result:")
        with open(c._files.final, "wb") as fh:
            pickle.dump({"max_stress_pa": 1.0}, fh)
        assert c.poll() == ("done", {"max_stress_pa": 1.0})
        assert c.poll() == ("running", 1.0)          # delivered once
    finally:
        root = c._files.root
        c.cleanup()
        assert not os.path.exists(root)
        c.cleanup()                                  # idempotent


def test_error_phase_falls_back_to_log():
    c = _client_with_files()
    try:
        _status(c, phase="error", error="No supports")
        assert c.poll() == ("error", "No supports")
        with open(c._files.log, "w") as fh:
            fh.write("trace\n")
        _status(c, phase="error")
        assert c.poll() == ("error", "trace")
    finally:
        c.cleanup()


def test_worker_exit_without_status_reports_log():
    c = _client_with_files()
    try:
        with open(c._files.log, "w") as fh:
            fh.write("boom")
        c._proc = subprocess.Popen([sys.executable, "-c", "pass"])
        c._proc.wait()
        assert c.poll() == ("error", "boom")
        os.remove(c._files.log)
        assert c.poll() == ("error", "worker exited early")
    finally:
        c.cleanup()


def test_wait_times_out_while_running():
    c = _client_with_files()
    try:
        assert c.wait(timeout=0.2, interval=0.05) == ("error", "timeout")
    finally:
        c.cleanup()
