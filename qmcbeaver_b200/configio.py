"""Configuration files (.cfgs) in the reference's format, and the
print_configs driver that writes them from device steps.

QMCConfigIO (QMcBeaver/src/QMCConfigIO.cpp:271-505) stores one record per
call of writeCorrelatedSamplingConfiguration: the electron count, the
positions R[N][3], lap(D)/D (Slater part, both spins), grad(D)/D [N][3],
ln J, the potential energy and a weight.  The reference writes binary
records (native int32 and float64, no padding; `inBinary = true`,
QMcBeaver/src/QMCConfigIO.cpp:26) and can write a text form for debugging
(fixed notation, 10 decimals, :349-381).  With print_configs 1 every
walker writes two records at every print_config_frequency-th iteration
after equilibration: the trial configuration with weight p (the acceptance
probability) and the original one with weight 1 - p
(QMcBeaver/src/QMCManager.cpp:797-799, QMcBeaver/src/QMCWalker.cpp:238-250);
QMCReadAndEvaluateConfigs reads them back for correlated-sampling parameter
optimisation (QMcBeaver/src/QMCReadAndEvaluateConfigs.cpp:176-230).
"""
from __future__ import annotations

import io
from typing import Dict, Iterator, Optional

import numpy as np

FIELDS = ("R", "D1", "D2", "lnJ", "PE", "weight")


def record_dtype(n_electrons: int) -> np.dtype:
    """One binary record (little-endian, packed)."""
    N = int(n_electrons)
    return np.dtype([("n", "<i4"), ("R", "<f8", (N, 3)), ("D1", "<f8"), ("D2", "<f8", (N, 3)), ("lnJ", "<f8"),
                     ("PE", "<f8"), ("weight", "<f8")])


def records_from_flat(flat: np.ndarray, n_electrons: int) -> np.ndarray:
    """Device records [k][6N + 4] (qmcb_run_step_configs) as structured records."""
    N = int(n_electrons)
    flat = np.asarray(flat, np.float64).reshape(-1, 6 * N + 4)
    out = np.zeros(len(flat), record_dtype(N))
    out["n"] = N
    out["R"] = flat[:, :3 * N].reshape(-1, N, 3)
    out["D1"] = flat[:, 3 * N]
    out["D2"] = flat[:, 3 * N + 1:6 * N + 1].reshape(-1, N, 3)
    out["lnJ"] = flat[:, 6 * N + 1]
    out["PE"] = flat[:, 6 * N + 2]
    out["weight"] = flat[:, 6 * N + 3]
    return out


class ConfigIO:
    """Writes or reads one configuration file, as QMCConfigIO does
    (open / writeCorrelatedSamplingConfiguration /
    readCorrelatedSamplingConfiguration / eof / close)."""

    def __init__(self, n_electrons: int, binary: bool = True):
        self.N = int(n_electrons)
        self.binary = binary
        self.dtype = record_dtype(self.N)
        self.fh: Optional[io.IOBase] = None
        self.writing = True
        self.num_written = 0
        self.num_read = 0

    def open(self, name: str, for_writing: bool) -> None:
        self.close()
        self.writing = for_writing
        if for_writing:
            self.num_written = 0
        mode = ("wb" if for_writing else "rb") if self.binary else ("w" if for_writing else "r")
        self.fh = open(name, mode)

    def close(self) -> None:
        if self.fh is not None:
            self.fh.close()
            self.fh = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    # ---------------------------------------------------------------- writing
    def write(self, R, D1, D2, lnJ, PE, weight) -> None:
        """One record (writeCorrelatedSamplingConfiguration)."""
        rec = np.zeros(1, self.dtype)
        rec["n"], rec["R"], rec["D1"], rec["D2"] = self.N, R, D1, D2
        rec["lnJ"], rec["PE"], rec["weight"] = lnJ, PE, weight
        self.write_records(rec)

    def write_records(self, recs: np.ndarray) -> None:
        """Many records at once (structured, record_dtype)."""
        if not self.writing or self.fh is None:
            raise IOError("configuration file is not open for writing")
        recs = np.asarray(recs, self.dtype)
        if self.binary:
            self.fh.write(recs.tobytes())
        else:
            for r in recs:
                self.fh.write(_text_record(r, self.N))
        self.num_written += len(recs)

    # ---------------------------------------------------------------- reading
    def read_all(self) -> np.ndarray:
        """Every remaining record."""
        if self.writing or self.fh is None:
            raise IOError("configuration file is not open for reading")
        if self.binary:
            data = self.fh.read()
            if len(data) % self.dtype.itemsize:
                raise IOError(f"truncated configuration file: {len(data)} bytes, records of {self.dtype.itemsize}")
            recs = np.frombuffer(data, self.dtype).copy()
            bad = recs["n"] != self.N
            if bad.any():
                raise IOError(f"record {int(np.argmax(bad))} holds {int(recs['n'][bad][0])} electrons, not {self.N}")
        else:
            recs = _parse_text(self.fh.read(), self.N, self.dtype)
        self.num_read += len(recs)
        return recs

    def __iter__(self) -> Iterator[np.void]:
        return iter(self.read_all())


def _text_record(r, N: int) -> str:
    f = lambda x: f"{x:.10f}"
    out = ["&", f"R\t{N}"]
    for i in range(N):
        out.append(f"\t{i}\t" + "\t".join(f(v) for v in r["R"][i]))
    out += ["D1", "\t" + f(r["D1"]), "D2"]
    for i in range(N):
        out.append("".join("\t" + f(v) for v in r["D2"][i]))
    out += ["lnJ\t", "\t" + f(r["lnJ"]), "PE\t", "\t" + f(r["PE"]), "W\t", "\t" + f(r["weight"])]
    return "\n".join(out) + "\n"


def _parse_text(text: str, N: int, dtype) -> np.ndarray:
    # the reader skips the three tokens "&", "R", N, then index + x y z per
    # electron, a label before each scalar block (QMcBeaver/src/QMCConfigIO.cpp:449-490)
    tok = text.split()
    per = 3 + 4 * N + 2 + 1 + 3 * N + 2 + 2 + 2
    if len(tok) % per:
        raise IOError("truncated text configuration file")
    recs = np.zeros(len(tok) // per, dtype)
    for k in range(len(recs)):
        t = tok[k * per:(k + 1) * per]
        recs[k]["n"] = N
        p = 3
        recs[k]["R"] = np.array([[float(t[p + 4 * i + j]) for j in (1, 2, 3)] for i in range(N)])
        p += 4 * N
        recs[k]["D1"] = float(t[p + 1])
        p += 3
        recs[k]["D2"] = np.array([float(x) for x in t[p:p + 3 * N]]).reshape(N, 3)
        p += 3 * N
        recs[k]["lnJ"] = float(t[p + 1])
        recs[k]["PE"] = float(t[p + 3])
        recs[k]["weight"] = float(t[p + 5])
    return recs


def read_configs(path: str, n_electrons: int, binary: bool = True) -> np.ndarray:
    io_ = ConfigIO(n_electrons, binary)
    io_.open(path, False)
    try:
        return io_.read_all()
    finally:
        io_.close()


def run_with_configs(functions, path: str, first_step: int, n_steps: int, frequency: int = 50,
                     binary: bool = True) -> Dict[str, float]:
    """Runs steps first_step .. first_step + n_steps - 1 on a
    QMCB200Functions handle and writes the configuration records of every
    step whose number is a multiple of `frequency` (print_configs 1,
    print_config_frequency), the other steps batched on the device.
    Returns the accumulated step statistics."""
    if frequency <= 0:
        raise ValueError("print_config_frequency must be positive")
    N = functions.N
    tot = {"sum_weight": 0.0, "sum_weight_energy": 0.0, "sum_accept": 0.0, "n_moves": 0.0, "records": 0}
    out = ConfigIO(N, binary)
    out.open(path, True)

    def add(st):
        tot["sum_weight"] += st.sum_weight
        tot["sum_weight_energy"] += st.sum_weight_energy
        tot["sum_accept"] += st.sum_accept
        tot["n_moves"] += st.n_moves

    try:
        step, end = first_step, first_step + n_steps
        while step < end:
            nxt = step if step % frequency == 0 else min(end, step + (frequency - step % frequency))
            if nxt > step:
                add(functions.run_steps(step, nxt - step))
                step = nxt
                continue
            flat, st = functions.run_step_configs(step)
            add(st)
            recs = records_from_flat(flat, N)
            out.write_records(recs)
            tot["records"] += len(recs)
            step += 1
    finally:
        out.close()
    return tot
