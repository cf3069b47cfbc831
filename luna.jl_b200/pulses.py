"""Input pulses of the high-level interface (the ``Pulses`` module of Luna.jl's
``src/Interface.jl:14-180``): a time-domain field (``fields.PulseField``) together with the
mode it is launched in and its polarisation. A list of them is the ``pulses`` argument of
``interface.prop_capillary_args`` (several pulses, e.g. two colours, each with its own mode
and polarisation)."""
from . import fields


class Pulse:
    """A pulse: ``field`` (a ``fields.PulseField``), ``mode`` ("lowest" or a mode name such
    as "HE12") and ``polarisation`` ("linear", "x", "y", "circular" or an ellipticity)."""

    def __init__(self, field, mode="lowest", polarisation="linear"):
        self.field, self.mode, self.polarisation = field, mode, polarisation


def GaussPulse(*, λ0, τfwhm, energy=None, power=None, ϕ=(), m=1, mode="lowest", polarisation="linear"):
    """``Pulses.GaussPulse`` (Interface.jl:57-90): a (super-)Gaussian pulse."""
    return Pulse(fields.GaussField(λ0, τfwhm, energy=energy, power=power, m=m, ϕ=ϕ), mode, polarisation)


def SechPulse(*, λ0, τfwhm=None, τw=None, energy=None, power=None, ϕ=(), mode="lowest",
              polarisation="linear"):
    """``Pulses.SechPulse`` (Interface.jl:92-124): a sech² pulse of FWHM ``τfwhm`` or
    natural width ``τw``."""
    return Pulse(fields.SechField(λ0, τfwhm=τfwhm, τw=τw, energy=energy, power=power, ϕ=ϕ), mode, polarisation)
