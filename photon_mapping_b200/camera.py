"""Camera and Image: the reference's pinhole camera (camera.h:10-48) and
float RGB image (image.h:10-91)."""
from __future__ import annotations

import ctypes as C
import math

import numpy as np

F = np.float32


def _normalize(v: np.ndarray) -> np.ndarray:
    ln = np.sqrt(F((v[0] * v[0] + v[1] * v[1]) + v[2] * v[2]))
    return (v / ln).astype(F)


def _cross(a: np.ndarray, b: np.ndarray) -> np.ndarray:
    return np.array([a[1] * b[2] - a[2] * b[1], a[2] * b[0] - a[0] * b[2],
                     a[0] * b[1] - a[1] * b[0]], F)


class PMCamera(C.Structure):
    _fields_ = [("position", C.c_float * 3), ("forward", C.c_float * 3),
                ("right", C.c_float * 3), ("up", C.c_float * 3), ("focal_length", C.c_float)]


class Camera:
    """camera.h:21-37: right = normalize(forward x (0,1,0)), up =
    normalize(right x forward), focal_length = 1 / tan(FOV / 2), in float."""

    def __init__(self, position, forward, FOV: float = 0.5 * 3.14159265359):
        self.position = np.asarray(position, F)
        self.forward = np.asarray(forward, F)
        self.right = _normalize(_cross(self.forward, np.array([0, 1, 0], F)))
        self.up = _normalize(_cross(self.right, self.forward))
        self.focal_length = F(1.0) / np.tan(F(0.5) * F(FOV))

    def sampleRay(self, uv):  # camera.h:41-47
        pin = self.position + self.focal_length * self.forward
        sensor = (self.position + F(uv[0]) * self.right) + F(uv[1]) * self.up
        return sensor.astype(F), _normalize((pin - sensor).astype(F)), 1.0

    def as_struct(self) -> PMCamera:
        c = PMCamera()
        c.position[:] = self.position.tolist()
        c.forward[:] = self.forward.tolist()
        c.right[:] = self.right.tolist()
        c.up[:] = self.up.tolist()
        c.focal_length = float(self.focal_length)
        return c

    def as_array(self) -> np.ndarray:
        return np.concatenate([self.position, self.forward, self.right, self.up,
                               [self.focal_length]]).astype(F)


class Image:
    """image.h: float RGB pixels, row-major, index 3*j + 3*width*i."""

    def __init__(self, width: int, height: int, pixels: np.ndarray | None = None):
        self.width, self.height = int(width), int(height)
        self.pixels = (np.zeros((self.height, self.width, 3), F) if pixels is None
                       else np.asarray(pixels, F).reshape(self.height, self.width, 3).copy())

    def getPixel(self, i, j):
        return self.pixels[i, j].copy()

    def addPixel(self, i, j, rgb):
        self.pixels[i, j] += np.asarray(rgb, F)

    def setPixel(self, i, j, rgb):
        self.pixels[i, j] = np.asarray(rgb, F)

    def divide(self, k: float):  # image.h:49-56
        self.pixels = (self.pixels / F(k)).astype(F)

    def gammaCorrection(self, gamma: float):  # image.h:58-67
        self.pixels = np.power(self.pixels, F(1.0) / F(gamma)).astype(F)

    def writePFM(self, filename: str):
        """Raw linear radiance as a little-endian colour PFM ("PF", scale
        -1), rows stored bottom to top as the format defines. The reference
        writes only clamped 8-bit PPM (image.h:69-90); PFM keeps the float
        values for comparisons such as the image error against the path
        tracer."""
        with open(filename, "wb") as f:
            f.write(f"PF\n{self.width} {self.height}\n-1.0\n".encode("ascii"))
            f.write(np.ascontiguousarray(self.pixels[::-1], dtype="<f4").tobytes())

    @classmethod
    def readPFM(cls, filename: str) -> "Image":
        """Reads a colour PFM written by writePFM (or any little- or
        big-endian "PF" file)."""
        with open(filename, "rb") as f:
            data = f.read()
        parts, pos = [], 0
        while len(parts) < 4:  # "PF", width, height, scale (whitespace separated)
            while data[pos:pos + 1].isspace():
                pos += 1
            end = pos
            while not data[end:end + 1].isspace():
                end += 1
            parts.append(data[pos:end].decode("ascii"))
            pos = end
        pos += 1  # the single whitespace byte after the scale
        if parts[0] != "PF":
            raise ValueError(f"{filename}: not a colour PFM file")
        w, h, scale = int(parts[1]), int(parts[2]), float(parts[3])
        dt = "<f4" if scale < 0 else ">f4"
        px = np.frombuffer(data, dtype=dt, count=w * h * 3, offset=pos).reshape(h, w, 3)
        return cls(w, h, px[::-1].astype(F))

    def writePPM(self, filename: str):  # image.h:69-90 (P3, clamped to 0..255)
        v = (F(255.0) * self.pixels)
        with np.errstate(invalid="ignore"):
            q = np.where(np.isfinite(v) & (v > 0), np.minimum(v, 4294967295.0), 0)
        q = np.minimum(q.astype(np.uint64), 255)
        with open(filename, "w") as f:
            f.write(f"P3\n{self.width} {self.height}\n255\n")
            f.write("".join(f"{r} {g} {b}\n" for r, g, b in q.reshape(-1, 3).tolist()))
