"""Reader and runner for the reference-oracle driver (TEST INFRASTRUCTURE ONLY).

The oracle driver (``oracle/ref_driver.c``) links the reference ccfd sources
unmodified and writes a small binary dump:  magic ``CCFDDMP1`` followed by
records ``char name[32]; int32 type (0 f64, 1 i64); int32 pad; int64 count;
data``.  Only tests, ``__graft_entry__.smoke()`` and the CPU-baseline leg of
``bench.py`` use this module, as the checker or the timed reference -- never as
the product path.
"""
from __future__ import annotations

import os
import subprocess
import tempfile

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
REF_DIR = os.path.join(_HERE, "_ref")


def ref_binary(eqn: str = "euler", fast: bool = False) -> str:
    """Path of the compiled reference driver for an equation system."""
    name = f"ccfd_ref_{eqn}" + ("_fast" if fast else "")
    return os.path.join(REF_DIR, name)


def have_ref(eqn: str = "euler", fast: bool = False) -> bool:
    return os.access(ref_binary(eqn, fast), os.X_OK)


def read_dump(path: str) -> dict:
    out = {}
    with open(path, "rb") as f:
        if f.read(8) != b"CCFDDMP1":
            raise ValueError(f"{path}: not an oracle dump")
        while True:
            name = f.read(32)
            if len(name) < 32:
                break
            hdr = np.frombuffer(f.read(8), dtype=np.int32)
            cnt = int(np.frombuffer(f.read(8), dtype=np.int64)[0])
            dt = np.float64 if hdr[0] == 0 else np.int64
            data = np.frombuffer(f.read(8 * cnt), dtype=dt).copy()
            out[name.rstrip(b"\0").decode()] = data
    return out


def run_ref(ini_text: str, mode: str, *args, eqn: str = "euler",
            fast: bool = False, state: np.ndarray | None = None,
            threads: int | None = None, workdir: str | None = None,
            files: dict | None = None, timeout: float = 3600.0,
            output: bool = False, rel_abort: float | None = None,
            vector: np.ndarray | None = None, ser_cfl_max: float | None = None) -> dict:
    """Run the reference driver on an .ini text in a scratch directory.

    ``state`` (N x 4 primitive states in reference cell order) replaces the
    initial condition.  ``files`` maps names to paths linked into the scratch
    directory (the reference's parser drops '/' from values, so a mesh file
    must sit in its working directory).  ``output``: the run ends with the
    reference's dataOutput; its files come back as ``out["output_files"]``
    ({name: text}).  ``vector`` (N x 4, cell order) is passed after the
    state file (mode ``jacobian``: the right-hand side of LUSGS).
    ``ser_cfl_max``: switched-evolution-relaxation CFL cap of the driver's
    time loop.  Returns the parsed dump.
    """
    exe = ref_binary(eqn, fast)
    if not os.access(exe, os.X_OK):
        raise FileNotFoundError(exe)
    with tempfile.TemporaryDirectory(dir=workdir) as tmp:
        for name, src in (files or {}).items():
            os.symlink(os.path.abspath(src), os.path.join(tmp, name))
        ini = os.path.join(tmp, "case.ini")
        with open(ini, "w") as f:
            f.write(ini_text)
        dump = os.path.join(tmp, "out.dump")
        argv = [exe, ini, dump, mode] + [str(a) for a in args]
        if state is not None:
            sp = os.path.join(tmp, "state.bin")
            np.ascontiguousarray(state, dtype=np.float64).tofile(sp)
            if len(args) == 0:
                argv.append("0")
            argv.append(sp)
        if vector is not None:
            vp = os.path.join(tmp, "vector.bin")
            np.ascontiguousarray(vector, dtype=np.float64).tofile(vp)
            if state is None:
                argv.append("-")
            argv.append(vp)
        env = dict(os.environ)
        if threads is not None:
            env["OMP_NUM_THREADS"] = str(threads)
        env.setdefault("OMP_NUM_THREADS", "1")
        if output:
            env["CCFD_REF_OUTPUT"] = "1"
        if rel_abort is not None:
            env["CCFD_REF_REL_ABORT"] = repr(float(rel_abort))
        if ser_cfl_max is not None:
            env["CCFD_REF_SER_CFL_MAX"] = repr(float(ser_cfl_max))
        r = subprocess.run(argv, cwd=tmp, env=env, capture_output=True,
                           text=True, timeout=timeout)
        if r.returncode != 0:
            raise RuntimeError(f"reference driver failed ({r.returncode}):\n"
                               f"{r.stdout[-3000:]}\n{r.stderr[-3000:]}")
        out = read_dump(dump)
        # error norms printed by calcErrors (src/analyze.c:506-513)
        rows = [ln.split(":", 1)[1].split() for ln in r.stdout.splitlines()
                if ln.startswith(("| L1  :", "| L2  :", "| Linf:"))]
        if len(rows) >= 3:
            out["errors_printed"] = np.array(rows[-3:], dtype=np.float64)
        # pressure-coefficient files written by calcCoef (src/analyze.c:
        # 302-367), as arrays of (x, y, phi, cp) rows
        if output:
            out["output_files"] = {}
            for name in sorted(os.listdir(tmp)):
                if name.endswith((".csv", ".curve", ".dem")) and "_CP_" not in name:
                    with open(os.path.join(tmp, name)) as f:
                        out["output_files"][name] = f.read()
        for name in sorted(os.listdir(tmp)):
            if "_CP_" in name and name.endswith(".csv"):
                side = "cp_pressure" if "pressureSide" in name else "cp_suction"
                out[side] = np.genfromtxt(os.path.join(tmp, name), delimiter=",",
                                          skip_header=1).reshape(-1, 4)
        return out
