"""save_state / load_state in ImmersedBodies.jl's binary layout (src/io/io.jl:1-71).

Layout: the 28-byte header "@ImmersedBodies.jl State v1@", index (Int64),
t0 (Float64), then q, q0, Γ, ψ, nonlin[1], nonlin[2], xb, ds, ub, F̃b as raw
column-major Float64, then freestream_vel (2 x Float64); little-endian.
A checkpoint written by either solver resumes on the other.
"""
from __future__ import annotations

import io as _io
import struct

import numpy as np

from .problem import Problem, State, set_time_index_, update_vars_

STATE_FILE_HEADER = b"@ImmersedBodies.jl State v1@"


def _arrays(state: State):
    return [state.q, state.q0, state.Gamma, state.psi, *state.nonlin, state.panels.xb, state.panels.ds,
            state.panels.ub, state.Fbt]


def save_state(f, state: State):
    """save_state(filename_or_io, state) (io.jl:10-25)."""
    if isinstance(f, (str, bytes)) or hasattr(f, "__fspath__"):
        with open(f, "wb") as fh:
            return save_state(fh, state)
    f.write(STATE_FILE_HEADER)
    f.write(struct.pack("<qd", state.index, state.t0))
    for a in _arrays(state):
        f.write(np.asarray(a, dtype="<f8").tobytes(order="F"))
    f.write(struct.pack("<dd", *state.freestream_vel))


def load_state_(f, state: State) -> State:
    """load_state!(filename_or_io, state) (io.jl:42-71)."""
    if isinstance(f, (str, bytes)) or hasattr(f, "__fspath__"):
        with open(f, "rb") as fh:
            return load_state_(fh, state)
    if f.read(len(STATE_FILE_HEADER)) != STATE_FILE_HEADER:
        raise ValueError("State file is missing header")
    index, t0 = struct.unpack("<qd", f.read(16))
    state.t0 = t0
    set_time_index_(state, index)
    for a in _arrays(state):
        buf = f.read(a.size * 8)
        a[...] = np.frombuffer(buf, dtype="<f8").reshape(a.shape, order="F")
    state.freestream_vel = struct.unpack("<dd", f.read(16))
    update_vars_(state)
    return state


def load_state(f, prob: Problem) -> State:
    """load_state(filename_or_io, prob) (io.jl:34)."""
    return load_state_(f, State(prob))


def state_bytes(state: State) -> bytes:
    b = _io.BytesIO()
    save_state(b, state)
    return b.getvalue()
