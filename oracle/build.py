"""Build the oracle (test infrastructure only) and stage the reference plugin.

* ``oracle/jla_oracle.c`` -> ``oracle/_build/libjla_oracle.so`` (gcc, -O2).
* When the reference checkout is mounted (``/root/reference``), its shipped
  precompiled Linux plugin ``fevc/fevc_rust_linux_x64.plugin`` is copied to
  ``oracle/_ref/`` so that the CPU-baseline leg of the benchmark can time the
  reference's own implementation on a machine without the checkout.  The copy
  is byte-for-byte; it is only loaded with dlopen and called through its
  documented C ABI.
"""

from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

HERE = Path(__file__).resolve().parent
BUILD = HERE / "_build"
REF_DIR = HERE / "_ref"
ORACLE_LIB = BUILD / "libjla_oracle.so"
REFERENCE_PLUGIN_SOURCE = Path("/root/reference/fevc/fevc_rust_linux_x64.plugin")
REFERENCE_PLUGIN = REF_DIR / "fevc_rust_linux_x64.plugin"


def build() -> Path:
    BUILD.mkdir(exist_ok=True)
    src = HERE / "jla_oracle.c"
    if not ORACLE_LIB.exists() or ORACLE_LIB.stat().st_mtime < src.stat().st_mtime:
        tmp = ORACLE_LIB.with_suffix(".tmp")
        subprocess.run(["gcc", "-O2", "-fPIC", "-shared", "-std=gnu11", str(src), "-o", str(tmp), "-lm"], check=True)
        tmp.replace(ORACLE_LIB)
    if REFERENCE_PLUGIN_SOURCE.exists():
        REF_DIR.mkdir(exist_ok=True)
        if not REFERENCE_PLUGIN.exists() or REFERENCE_PLUGIN.stat().st_size != REFERENCE_PLUGIN_SOURCE.stat().st_size:
            shutil.copyfile(REFERENCE_PLUGIN_SOURCE, REFERENCE_PLUGIN)
    return ORACLE_LIB


if __name__ == "__main__":
    print(build())
