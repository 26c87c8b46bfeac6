"""The reference's own CPU runner (oracle/_ref/libes_refrun.so, test
infrastructure only): runs a .config through SimulationRunner::Run
(src/SimulationRunner.cpp:32-52) in a child process.

The reference writes Metrics.txt through a wide stream imbued with the
en_US.UTF-8 locale (src/Logger.cpp:142), which this image does not install
(only C, C.utf8 and POSIX exist), so std::locale's constructor would throw. The
child runs with LOCPATH pointing at a directory where the name en_US.UTF-8
holds a copy of the image's own C.utf8 locale: UTF-8 output of the box-drawing
characters, and C's numeric punctuation (no digit grouping)."""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
import tempfile
from pathlib import Path

ROOT = Path(__file__).resolve().parent.parent
REFRUN_SO = ROOT / "oracle" / "_ref" / "libes_refrun.so"
C_UTF8 = Path("/usr/lib/locale/C.utf8")


def available() -> bool:
    return REFRUN_SO.exists() and C_UTF8.is_dir()


def run(config_path: Path, cwd: Path, timeout: float = 600.0) -> subprocess.CompletedProcess:
    locdir = Path(tempfile.mkdtemp(prefix="es_locale_"))
    try:
        shutil.copytree(C_UTF8, locdir / "en_US.UTF-8")
        env = dict(os.environ, LOCPATH=str(locdir))
        code = ("import ctypes, sys; lib = ctypes.CDLL(sys.argv[1]); "
                "lib.refrun.argtypes = [ctypes.c_char_p]; sys.exit(lib.refrun(sys.argv[2].encode()))")
        return subprocess.run([sys.executable, "-c", code, str(REFRUN_SO), str(config_path)], cwd=cwd, env=env,
                              capture_output=True, text=True, timeout=timeout)
    finally:
        shutil.rmtree(locdir, ignore_errors=True)
