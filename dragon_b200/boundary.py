"""Ghost-fill API mirroring DRAGON's Boundary namespace.

Same names, arguments and composition rules as the reference
(DRAGON/Boundary/Boundary.hpp:119-229, BoundaryList.hpp:22-128): elements
combine with ``+`` into a BoundaryList applied in order, after an implicit
Outflow over every face no element covers. The list is compiled into
dragon_bc_desc records and executed on the device.

Example (the reference's ``Boundary::Reflective("X") + Boundary::Periodic("YZ")``)::

    grid.boundary = Reflective("X") + Periodic("YZ")
"""
from __future__ import annotations

import ctypes

from typing import Iterable, Sequence

# Face bits (Boundary.hpp:139-149)
X_negative = 1 << 0
X_positive = 1 << 1
X = X_negative | X_positive
Y_negative = 1 << 2
Y_positive = 1 << 3
Y = Y_negative | Y_positive
Z_negative = 1 << 4
Z_positive = 1 << 5
Z = Z_negative | Z_positive

OUTFLOW, OUTFLOW_GATED, FIXED, REFLECTIVE, PERIODIC, IGNORE, USER = range(7)


def face_mask(s: str) -> int:
    """Boundary::face_mask (GhostFill.cpp:14-48): "X", "X-", "YZ+", "L/R/U/D"."""
    mask = 0
    s = s + " "
    for cur, nxt in zip(s, s[1:]):
        c = cur.upper()
        if c in "XYZ":
            neg, pos, both = {"X": (X_negative, X_positive, X), "Y": (Y_negative, Y_positive, Y),
                              "Z": (Z_negative, Z_positive, Z)}[c]
            mask |= pos if nxt == "+" else (neg if nxt == "-" else both)
        elif c == "L":
            mask |= X_negative
        elif c == "R":
            mask |= X_positive
        elif c == "U":
            mask |= Y_positive
        elif c == "D":
            mask |= Y_negative
    return mask


def _faces(f) -> int:
    return face_mask(f) if isinstance(f, str) else int(f)


class GhostFill:
    """A boundary element (GhostFill.hpp:16-30): face mask + corner flag."""

    kind = IGNORE

    def __init__(self, faces=X | Y | Z, corner_ghosts: bool = True):
        self.faces = _faces(faces)
        self.corners = bool(corner_ghosts)

    def get_faces(self) -> int:
        return self.faces

    def state(self) -> Sequence[float]:
        return ()

    # Interior layers next to its faces a user element reads (None: the ghost
    # width). Only these and the ghost layers of its faces cross the host link.
    reach = None

    def apply(self, grid) -> None:
        """GhostFill::apply(Grid&) (GhostFill.hpp:16-30). A user element
        subclasses GhostFill and overrides this to fill grid's ghost cells on
        the host (grid.w / grid.B, or grid[i, j] with ghost coordinates), like
        the reference's Jet (Jets.hpp:12-39). Grids then run such lists on the
        host-driven path: the built-in elements stay on the device, and around
        each user element only the slabs along its faces cross to the host and
        back: its ghost layers and `reach` interior layers next to them, over
        the whole transverse extent (corners included). apply must read and
        write inside those slabs."""
        raise NotImplementedError(f"{type(self).__name__} is a built-in element applied on the device")

    @property
    def is_custom(self) -> bool:
        return type(self).apply is not GhostFill.apply

    def __add__(self, other):
        return BoundaryList(self) + other

    def __radd__(self, other):
        if other == 0:
            return BoundaryList(self)
        return NotImplemented

    def __repr__(self):
        return f"{type(self).__name__}(faces={self.faces}, corners={self.corners})"


class DeviceGhostFill(GhostFill):
    """A user element (GhostFill.hpp:16-30) whose fill runs on the device.

    `source` is CUDA C++ defining ``__device__ void <function>(const
    dragon_fill_ctx& c, int i, int j, int k)``, called once per ghost cell of
    `fill_faces` (the faces whose ghost layers it fills; default its own
    `faces` mask) with c.get / c.set (primitive fields DRAGON_RHO, DRAGON_P,
    DRAGON_VX.. , DRAGON_BX..), c.getB / c.setB (face B), c.n, c.g, c.d,
    c.axis / c.side and c.params (`params`); include/dragon_gpu.h gives the
    contract. It is compiled once with NVRTC and the grid launches it at the
    element's place in the list inside the device advance loop, so unlike a
    host `apply` no state crosses the host link. `faces` keeps its
    BoundaryList meaning: the faces the element claims (the reference's Jet
    claims none, GhostFill(0, true), and fills its jet face over the implicit
    Outflow)."""

    kind = USER
    _compiled = {}

    def __init__(self, source: str, function: str, faces=0, corner_ghosts: bool = True, fill_faces=None,
                 params: Sequence[float] = ()):
        super().__init__(faces, corner_ghosts)
        self.fill_faces = self.faces if fill_faces is None else _faces(fill_faces)
        self.params = [float(v) for v in params]
        self.source, self.function = source, function
        self._fill = DeviceGhostFill.compile(source, function)

    @staticmethod
    def compile(source: str, function: str):
        """The compiled fill (a dragon_user_fill*), shared by every element
        with the same source and function."""
        key = (source, function)
        if key not in DeviceGhostFill._compiled:
            from . import _lib
            lib = _lib.load()
            out = ctypes.c_void_p()
            _lib.check(lib.dragon_gpu_user_fill_create(source.encode(), function.encode(), ctypes.byref(out)))
            DeviceGhostFill._compiled[key] = out
        return DeviceGhostFill._compiled[key]

    def bind(self, lib, handle, entry: int, fill_faces: int | None = None):
        """dragon_gpu_set_user_fill for list entry `entry` of a grid
        (fill_faces overrides the element's own, e.g. masked to the faces a
        slab of a distributed grid owns)."""
        from . import _lib
        arr = (ctypes.c_double * max(1, len(self.params)))(*self.params)
        ff = self.fill_faces if fill_faces is None else int(fill_faces)
        _lib.check(lib.dragon_gpu_set_user_fill(handle, entry, self._fill, ff, int(self.corners), arr,
                                                len(self.params)))


class Outflow(GhostFill):
    """Outflow (Outflow.cpp): ghosts copy the nearest interior cell; Gated
    variants zero inflowing normal velocity."""

    def __init__(self, faces=X | Y | Z, corner_ghosts: bool = True, gated: bool = False):
        super().__init__(faces, corner_ghosts)
        self.gated = bool(gated)

    @property
    def kind(self):
        return OUTFLOW_GATED if self.gated else OUTFLOW

    @staticmethod
    def Gated(faces=X | Y | Z, corner_ghosts: bool = True) -> "Outflow":
        return Outflow(faces, corner_ghosts, True)


class Fixed(GhostFill):
    """Fixed (Fixed.cpp): ghosts take a fixed primitive state
    (rho, p, vx, vy, vz[, Bx, By, Bz])."""

    kind = FIXED

    def __init__(self, state: Sequence[float], faces=X | Y | Z, corner_ghosts: bool = True):
        super().__init__(faces, corner_ghosts)
        st = [float(v) for v in state]
        if len(st) not in (5, 8):
            raise ValueError("Fixed state needs 5 (hydro) or 8 (MHD) primitive values")
        self._state = st + [0.0] * (8 - len(st))

    def state(self):
        return self._state


class Reflective(GhostFill):
    """Reflective (Reflective.cpp): mirrored cells, normal velocity flipped."""

    kind = REFLECTIVE


class Periodic(GhostFill):
    """Periodic (Periodic.cpp): either face of an axis selects both."""

    kind = PERIODIC

    def __init__(self, faces=X | Y | Z, corner_ghosts: bool = True):
        super().__init__(faces, corner_ghosts)
        f = self.faces
        self.faces = (X if f & X else 0) | (Y if f & Y else 0) | (Z if f & Z else 0)


class Ignore(GhostFill):
    """Ignore (Ignore.cpp): fills nothing but counts as covering its faces."""

    kind = IGNORE


class BoundaryList:
    """Ordered boundary elements plus the implicit Outflow (BoundaryList.hpp)."""

    def __init__(self, *elements: GhostFill):
        self.elements: list[GhostFill] = []
        for e in elements:
            self.append(e)

    def append(self, e) -> None:
        if isinstance(e, BoundaryList):
            self.elements.extend(e.elements)
        elif isinstance(e, GhostFill):
            self.elements.append(e)
        else:
            raise TypeError(f"not a boundary element: {e!r}")

    def prepend(self, e) -> None:
        if isinstance(e, BoundaryList):
            self.elements[:0] = e.elements
        else:
            self.elements.insert(0, e)

    def clear(self) -> None:
        self.elements.clear()

    def __add__(self, other):
        out = BoundaryList(*self.elements)
        out.append(other)
        return out

    def __radd__(self, other):
        out = BoundaryList()
        out.append(other)
        out.append(self)
        return out

    def __iadd__(self, other):
        self.append(other)
        return self

    def has_custom(self) -> bool:
        return any(e.is_custom for e in self.elements)

    def uncovered_faces(self) -> int:
        m = X | Y | Z
        for e in self.elements:
            m &= ~e.get_faces()
        return m

    def __iter__(self):
        return iter(self.elements)

    def __len__(self):
        return len(self.elements)

    def __repr__(self):
        return "BoundaryList(" + " + ".join(map(repr, self.elements)) + ")"


def as_list(b) -> BoundaryList:
    if b is None:
        return BoundaryList()
    if isinstance(b, BoundaryList):
        return b
    if isinstance(b, GhostFill):
        return BoundaryList(b)
    if isinstance(b, Iterable):
        return BoundaryList(*b)
    raise TypeError(f"cannot use {b!r} as a boundary")
