"""Host logic of the batched and served forms that needs no GPU: the
device-arena bookkeeping (lumenstereo_b200/csrc/host_arena.h) under a
randomised allocate/free sequence, the batched sweep launch's ticket table
(lumenstereo_b200/csrc/batch_tickets.h) against the ordering and window
properties its progress rests on, and the server's option defaults."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_arena_first_fit_and_coalescing(tmp_path):
    exe = tmp_path / "arena_test"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "lumenstereo_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "arena_test.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=120)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr


@pytest.mark.skipif(shutil.which("g++") is None, reason="needs g++")
def test_ticket_table_order_and_window(tmp_path):
    exe = tmp_path / "tickets_test"
    subprocess.run(["g++", "-std=c++17", "-O2", "-I", os.path.join(ROOT, "lumenstereo_b200", "csrc"),
                    os.path.join(ROOT, "tests", "cpp", "tickets_test.cpp"), "-o", str(exe)], check=True)
    out = subprocess.run([str(exe)], capture_output=True, text=True, timeout=300)
    assert out.returncode == 0 and out.stdout.strip() == "ok", out.stdout + out.stderr


def test_server_options_defaults():
    from lumenstereo_b200 import _lib
    try:
        lib = _lib.lib()
    except OSError:
        pytest.skip("library not built")
    o = _lib.CServerOptions()
    lib.lumen_server_options_default(o)
    assert o.device_budget_bytes == 40 << 30
    assert (o.max_batch_pairs, o.rows_per_band, o.max_inflight, o.watchdog_ms) == (32, 16, 2, 60000)
    assert o.plain_fallback == 1 and o.schedule == 6
