"""Event-chain Monte Carlo on the B200 library (qcb_ecmc_*, include/qcb.h).

    reference (C++, MPI, src/ecmc/ecmc_mpi_cb.h)            here
    ---------------------------------------------------------------------------------------
    LocalChainState (one per rank)                         one record per l_core^4 block
                                                             (CHAIN_DTYPE, EventChains.chains())
    ECMCParams (src/io/params.h:9-17)                      EcmcParams (+ l_core)
    mpi::ecmccb::sample_persistant(state, d, field, geo,   ecmccb.sample_persistant(chains, shift)
        params, rng) on every rank                           (every block's chain in one launch)

The chains of all blocks run at once on the GPU; the blocks follow the cumulative shift of
the field's random translations as qcb_heatbath_frozen does.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from ._lib import EcmcParams, check, lib

# qcb_ecmc_chain, 256 bytes
CHAIN_DTYPE = np.dtype([
    ("R", np.complex128, (3, 3)),
    ("theta_refresh_site", np.float64), ("theta_refresh_R", np.float64),
    ("travelled_site", np.float64), ("travelled_R", np.float64),
    ("draws", np.uint64), ("events", np.uint64), ("lifts", np.uint64), ("revs", np.uint64),
    ("site", np.int32, (4,)), ("mu", np.int32), ("epsilon", np.int32),
    ("initialized", np.int32), ("status", np.int32), ("set_counter", np.int32), ("pad", np.int32, (3,)),
])
assert CHAIN_DTYPE.itemsize == 256


def params(beta=6.0, theta_sample=100.0, theta_refresh_site=50.0, theta_refresh_R=15.0, epsilon_set=0.15,
           poisson=False, l_core=4) -> EcmcParams:
    """EcmcParams with the reference's ECMCParams defaults (src/io/params.h:9-17)."""
    return EcmcParams(float(beta), float(theta_sample), float(theta_refresh_site), float(theta_refresh_R),
                      float(epsilon_set), 1 if poisson else 0, int(l_core))


class EventChains:
    """The persistent chains of one lattice (qcb_ecmc): one chain per l_core^4 block."""

    def __init__(self, field, p: EcmcParams | dict, seed: int):
        if isinstance(p, dict):
            p = params(**p)
        h = C.c_void_p()
        check(lib().qcb_ecmc_create(field.h, C.byref(p), C.c_uint64(seed), C.byref(h)))
        self.h = h
        self.field = field
        self.params = p
        n = C.c_int()
        check(lib().qcb_ecmc_num_chains(self.h, C.byref(n)))
        self.n_chains = n.value
        field.ctx._adopt(self)

    @property
    def lanes(self) -> int:
        """Lanes of a warp per chain in the next call (1, 3 or 6)."""
        n = C.c_int()
        check(lib().qcb_ecmc_lanes(self.h, C.byref(n)))
        return n.value

    @lanes.setter
    def lanes(self, lanes: int) -> None:
        """1, 3 or 6 lanes per chain, or 0 to let the library choose; results are the same."""
        check(lib().qcb_ecmc_set_lanes(self.h, int(lanes)))

    def sample(self, shift=(0, 0, 0, 0)) -> None:
        """One sample call of every chain (asynchronous); shift = cumulative shift of the field."""
        check(lib().qcb_ecmc_sample(self.h, (C.c_int * 4)(*[int(s) for s in shift])))

    def sample_n(self, shifts) -> None:
        """Consecutive sample calls, one per row of cumulative shifts (n x 4), with one pack
        and one unpack of the lattice; the same result as sample() per row."""
        sh = np.ascontiguousarray(np.asarray(shifts, dtype=np.int32).reshape(-1, 4))
        check(lib().qcb_ecmc_sample_n(self.h, sh.ctypes.data_as(C.POINTER(C.c_int)), int(sh.shape[0])))

    def counters(self, reset: bool = False):
        """(events, lifts, same-site lifts) summed over the chains."""
        out = (C.c_uint64 * 3)()
        check(lib().qcb_ecmc_counters(self.h, out, 1 if reset else 0))
        return int(out[0]), int(out[1]), int(out[2])

    def chains(self):
        """(records, calls): a copy of the chain records and the number of sample calls made."""
        rec = np.zeros(self.n_chains, CHAIN_DTYPE)
        calls = C.c_uint64()
        check(lib().qcb_ecmc_get_chains(self.h, rec.ctypes.data_as(C.c_void_p), C.byref(calls)))
        return rec, calls.value

    def set_chains(self, records, calls: int) -> None:
        rec = np.ascontiguousarray(records, CHAIN_DTYPE)
        if rec.shape != (self.n_chains,):
            raise ValueError(f"expected {self.n_chains} chain records")
        check(lib().qcb_ecmc_set_chains(self.h, rec.ctypes.data_as(C.c_void_p), C.c_uint64(calls)))

    def close(self) -> None:
        if getattr(self, "h", None):
            lib().qcb_ecmc_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


class ecmccb:
    """mpi::ecmccb (src/ecmc/ecmc_mpi_cb.h:55-117)."""

    @staticmethod
    def sample_persistant(chains: EventChains, shift=(0, 0, 0, 0)) -> None:
        chains.sample(shift)
