"""Fenton-Karma parameter set (runtime, not compile-time).

The reference fixes the parameters with ``#define``s and ``constexpr h`` in
src/cuda/fk_parameters_00_05_alpha_0p8_dx_0p035.h:2-24, chosen by an external
``sed`` of the include line (src/cuda/fk_forward_Et_mono_PARAMETERS.cu:13-20).
Here they are one struct passed at run time; the defaults are that header's
values and ``h`` is the grid spacing (cm).
"""
from __future__ import annotations

import ctypes as C
from dataclasses import asdict, dataclass, fields, replace

FIELDS = ("u_c", "u_v", "tau_d", "tau_v1_minus", "tau_v2_minus", "tau_v_plus", "tau_0",
          "tau_r", "tau_si", "u_csi", "k_fk", "tau_w_minus", "tau_w_plus", "Du", "Dv", "Dw",
          "ksm", "h")


@dataclass(frozen=True)
class FkParams:
    u_c: float = 0.13
    u_v: float = 0.04
    tau_d: float = 0.388
    tau_v1_minus: float = 7.6
    tau_v2_minus: float = 8.8
    tau_v_plus: float = 3.324
    tau_0: float = 8.2
    tau_r: float = 33.264
    tau_si: float = 29.0
    u_csi: float = 0.54
    k_fk: float = 15.0
    tau_w_minus: float = 68.0
    tau_w_plus: float = 399.99999999999994
    Du: float = 1.0e-3
    Dv: float = 1.0e-5
    Dw: float = 1.0e-5
    ksm: float = 100.0
    h: float = 0.035

    def with_h(self, h: float) -> "FkParams":
        return replace(self, h=float(h))

    def as_dict(self) -> dict:
        return asdict(self)

    def describe(self) -> str:
        """Parameter provenance text (the role of the reference's param_str,
        src/cuda/fk_parameters_string_00_05_alpha_0p8_dx_0p035.cpp:1-32)."""
        return "".join(f"{f.name} = {getattr(self, f.name)!r}\n" for f in fields(self))


class CFkParams(C.Structure):
    """Mirror of ``fkadj_params`` in include/fkadj.h (18 doubles, this order)."""
    _fields_ = [(f, C.c_double) for f in FIELDS]

    @classmethod
    def of(cls, p: FkParams) -> "CFkParams":
        return cls(*[float(getattr(p, f)) for f in FIELDS])


assert tuple(f.name for f in fields(FkParams)) == FIELDS
