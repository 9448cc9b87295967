"""NCCL is opened by the library at run time, by soname, the first time a
communicator id is made.  The Python binding first loads the NCCL of the
nvidia-nccl wheel (the one PyTorch links), so that importing torch afterwards
still finds the NCCL symbols it needs: a system libnccl.so.2 opened first
would satisfy torch's own load of that soname.  Run in a fresh interpreter,
since the test process may already hold torch."""
import os
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

SCRIPT = """
import sys
sys.path.insert(0, %r)
from emu_b200 import api
api.comm_id()
import torch
print("ok")
""" % ROOT


def test_comm_id_then_torch_import():
    env = dict(os.environ)
    env.pop("EMU_NCCL_LIBRARY", None)
    r = subprocess.run([sys.executable, "-c", SCRIPT], capture_output=True, text=True, timeout=600, env=env)
    assert r.returncode == 0 and r.stdout.strip().endswith("ok"), r.stderr[-2000:]
