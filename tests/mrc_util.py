"""Small MRC writer/reader for the CLI tests (standard 1024-byte header)."""
import numpy as np

HDR = np.dtype([("nx", "<i4"), ("ny", "<i4"), ("nz", "<i4"), ("mode", "<i4"),
                ("start", "<i4", 3), ("m", "<i4", 3), ("len", "<f4", 3), ("ang", "<f4", 3),
                ("map", "<i4", 3), ("amin", "<f4"), ("amax", "<f4"), ("amean", "<f4"),
                ("ispg", "<i2"), ("nsymbt", "<i2"), ("next", "<i4"), ("creatid", "<i2"),
                ("blank", "S30"), ("nint", "<i2"), ("nreal", "<i2"), ("sub", "<i2"),
                ("zfac", "<i2"), ("mm", "<f4", 6), ("idtype", "<i2"), ("lens", "<i2"),
                ("nd", "<i2", 4), ("tilt", "<f4", 6), ("org", "<f4", 3), ("cmap", "S4"),
                ("stamp", "S4"), ("rms", "<f4"), ("nlabl", "<i4"), ("labels", "S800")])
assert HDR.itemsize == 1024


def write_mrc(path, data, mode=2, next_bytes=0):
    """data: [nz][ny][nx]."""
    data = np.asarray(data)
    h = np.zeros((), HDR)
    h["nz"], h["ny"], h["nx"] = data.shape
    h["mode"] = mode
    h["next"] = next_bytes
    dt = {0: np.int8, 1: np.int16, 2: np.float32}[mode]
    with open(path, "wb") as f:
        f.write(h.tobytes())
        f.write(b"\0" * next_bytes)
        f.write(np.ascontiguousarray(data, dt).tobytes())


def read_mrc(path):
    raw = open(path, "rb").read()
    h = np.frombuffer(raw[:1024], HDR)[0]
    dt = {0: np.uint8, 1: np.int16, 2: np.float32}[int(h["mode"])]
    off = 1024 + int(h["next"])
    n = int(h["nx"]) * int(h["ny"]) * int(h["nz"])
    data = np.frombuffer(raw[off:off + n * np.dtype(dt).itemsize], dt)
    return h, raw[:1024], data.reshape(int(h["nz"]), int(h["ny"]), int(h["nx"]))


def write_angles(path, angles):
    with open(path, "w") as f:
        f.write("\n".join(f"{a:.4f}" for a in angles) + "\n")
