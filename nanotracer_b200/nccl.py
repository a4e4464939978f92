"""NCCL through its C API (ctypes), for the data-parallel views path.

The collectives of one split iteration (multiview.py) run on the library
context's CUDA stream, so they are ordered with the library's kernels and
device copies without any other runtime in between.  The communicator's
unique id goes from rank 0 to the others over a plain TCP connection
(rendezvous_bytes), so no launcher or store is needed beyond an address and
a port every rank knows.

libnccl.so.2 is looked up in NANOTRACER_NCCL_LIB, then in the nvidia/nccl
wheel next to the Python packages, then on the system library path.
"""
from __future__ import annotations

import ctypes as C
import glob
import os
import socket
import struct
import sys
import time

NCCL_FLOAT32 = 7
NCCL_FLOAT64 = 8
NCCL_SUM = 0
UNIQUE_ID_BYTES = 128


class ncclUniqueId(C.Structure):
    _fields_ = [("internal", C.c_char * UNIQUE_ID_BYTES)]


class NcclError(RuntimeError):
    pass


_lib = None


def _candidates() -> list[str]:
    out = []
    if os.environ.get("NANOTRACER_NCCL_LIB"):
        out.append(os.environ["NANOTRACER_NCCL_LIB"])
    for p in sys.path:
        out += sorted(glob.glob(os.path.join(p, "nvidia", "nccl", "lib", "libnccl.so*")))
    out += ["libnccl.so.2", "libnccl.so"]
    return out


def lib():
    global _lib
    if _lib is None:
        errs = []
        for path in _candidates():
            try:
                L = C.CDLL(path, mode=C.RTLD_GLOBAL)
                break
            except OSError as e:
                errs.append(f"{path}: {e}")
        else:
            raise NcclError("libnccl.so.2 not found: " + "; ".join(errs))
        P, I, SZ = C.c_void_p, C.c_int, C.c_size_t
        protos = {
            "ncclGetUniqueId": (I, [C.POINTER(ncclUniqueId)]),
            "ncclCommInitRank": (I, [C.POINTER(P), I, ncclUniqueId, I]),
            "ncclCommDestroy": (I, [P]),
            "ncclCommAbort": (I, [P]),
            "ncclGetErrorString": (C.c_char_p, [I]),
            "ncclReduceScatter": (I, [P, P, SZ, I, I, P, P]),
            "ncclAllGather": (I, [P, P, SZ, I, P, P]),
            "ncclAllReduce": (I, [P, P, SZ, I, I, P, P]),
            "ncclGetVersion": (I, [C.POINTER(I)]),
        }
        for name, (res, args) in protos.items():
            f = getattr(L, name)
            f.restype, f.argtypes = res, args
        _lib = L
    return _lib


def _check(rc: int, what: str) -> None:
    if rc != 0:
        msg = lib().ncclGetErrorString(rc)
        raise NcclError(f"{what}: {msg.decode() if msg else rc}")


def version() -> int:
    v = C.c_int()
    _check(lib().ncclGetVersion(C.byref(v)), "ncclGetVersion")
    return v.value


def _recv_exact(sock: socket.socket, n: int) -> bytes:
    buf = b""
    while len(buf) < n:
        chunk = sock.recv(n - len(buf))
        if not chunk:
            raise NcclError("rendezvous: connection closed before the id arrived")
        buf += chunk
    return buf


def rendezvous_bytes(payload: bytes | None, rank: int, world: int, host: str, port: int,
                     timeout: float = 60.0) -> bytes:
    """Rank 0's `payload` (a fixed-size byte string) delivered to every rank:
    rank 0 listens on (host, port) and sends it to each of the world - 1
    connections; the others connect (retrying until `timeout`) and receive it.
    A peer that never arrives ends in an error after `timeout`, not a hang."""
    if world == 1:
        return payload
    deadline = time.time() + timeout
    if rank == 0:
        assert payload is not None
        with socket.socket(socket.AF_INET, socket.SOCK_STREAM) as srv:
            srv.setsockopt(socket.SOL_SOCKET, socket.SO_REUSEADDR, 1)
            srv.bind((host, port))
            srv.listen(world)
            for _ in range(world - 1):
                srv.settimeout(max(0.1, deadline - time.time()))
                try:
                    conn, _ = srv.accept()
                except socket.timeout as e:
                    raise NcclError(f"rendezvous: not every rank connected within {timeout:.0f} s") from e
                with conn:
                    conn.sendall(struct.pack("<I", len(payload)) + payload)
        return payload
    while True:
        try:
            with socket.create_connection((host, port), timeout=max(0.1, deadline - time.time())) as s:
                s.settimeout(max(0.1, deadline - time.time()))
                n = struct.unpack("<I", _recv_exact(s, 4))[0]
                return _recv_exact(s, n)
        except (ConnectionRefusedError, socket.timeout, OSError) as e:
            if time.time() > deadline:
                raise NcclError(f"rendezvous: rank 0 not reachable at {host}:{port}") from e
            time.sleep(0.05)


class NcclComm:
    """One rank of an NCCL communicator whose collectives run on `stream`
    (a cudaStream_t as an integer, e.g. CudaCtx.stream)."""

    def __init__(self, rank: int, world: int, stream: int, host: str = "127.0.0.1", port: int = 29500,
                 timeout: float = 60.0):
        self.rank, self.world, self.stream = rank, world, C.c_void_p(stream)
        uid = ncclUniqueId()
        payload = None
        if rank == 0:
            _check(lib().ncclGetUniqueId(C.byref(uid)), "ncclGetUniqueId")
            payload = bytes(C.string_at(C.addressof(uid), UNIQUE_ID_BYTES))
        data = rendezvous_bytes(payload, rank, world, host, port, timeout)
        C.memmove(C.addressof(uid), data, UNIQUE_ID_BYTES)
        self.comm = C.c_void_p()
        _check(lib().ncclCommInitRank(C.byref(self.comm), world, uid, rank), "ncclCommInitRank")

    # device pointers (integers); counts in elements
    def reduce_scatter_f32(self, recv: int, send: int, recv_count: int) -> None:
        _check(lib().ncclReduceScatter(C.c_void_p(send), C.c_void_p(recv), recv_count, NCCL_FLOAT32, NCCL_SUM,
                                       self.comm, self.stream), "ncclReduceScatter")

    def all_gather_f32(self, recv: int, send: int, send_count: int) -> None:
        _check(lib().ncclAllGather(C.c_void_p(send), C.c_void_p(recv), send_count, NCCL_FLOAT32, self.comm,
                                   self.stream), "ncclAllGather")

    def all_reduce_sum_f64(self, buf: int, count: int) -> None:
        _check(lib().ncclAllReduce(C.c_void_p(buf), C.c_void_p(buf), count, NCCL_FLOAT64, NCCL_SUM, self.comm,
                                   self.stream), "ncclAllReduce")

    def close(self, abort: bool = False) -> None:
        if self.comm:
            (lib().ncclCommAbort if abort else lib().ncclCommDestroy)(self.comm)
            self.comm = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass
