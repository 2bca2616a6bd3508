"""Reader of the TRZ trajectory layout that WRITETRJ.F90:50-95 writes (test
infrastructure): Fortran unformatted sequential records, each framed by 4-byte
length markers.  The file starts with an 80-character title record and a
record-count record; each frame is a header (frame, frame index, NATOMS, time
in ps), the 3x3 box (REAL*8), the pressure and pressure tensor (7 x REAL*8),
the energy record (an integer 6 and 6 x REAL*8), then x, y, z and vx, vy, vz
as NATOMS x REAL*4 each."""
import struct

import numpy as np


def records(path):
    data = open(path, "rb").read()
    at = 0
    while at < len(data):
        (n,) = struct.unpack_from("<i", data, at)
        payload = data[at + 4: at + 4 + n]
        (m,) = struct.unpack_from("<i", data, at + 4 + n)
        assert m == n, "record markers differ"
        yield payload
        at += 8 + n


def read_trz(path):
    rec = list(records(path))
    title = rec[0].decode().rstrip()
    (nrec,) = struct.unpack("<i", rec[1])
    frames = []
    k = 2
    while k < len(rec):
        nframe, index, natoms = struct.unpack_from("<3i", rec[k])
        (time_ps,) = struct.unpack_from("<d", rec[k], 12)
        box = np.frombuffer(rec[k + 1], "<f8").reshape(3, 3)
        press = np.frombuffer(rec[k + 2], "<f8")
        (six,) = struct.unpack_from("<i", rec[k + 3])
        energy = np.frombuffer(rec[k + 3][4:], "<f8")
        xyz = np.stack([np.frombuffer(rec[k + 4 + c], "<f4") for c in range(3)], 1)
        vel = np.stack([np.frombuffer(rec[k + 7 + c], "<f4") for c in range(3)], 1)
        frames.append({"frame": nframe, "index": index, "natoms": natoms, "time_ps": time_ps, "box": box,
                       "pressure": press, "n_energy": six, "energy": energy, "xyz": xyz, "vel": vel})
        k += 10
    return title, nrec, frames
