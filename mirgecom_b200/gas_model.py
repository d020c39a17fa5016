"""Gas model and fluid states, mirroring mirgecom/gas_model.py.

``make_fluid_state`` (mirgecom/gas_model.py:302-430) returns a
:class:`FluidState` holding the conserved state and its temperature.  For a
mixture the temperature is the fixed-count Newton solve seeded with
*temperature_seed*; the same launch also produces the temperature the
operator states carry (the reference re-solves every operator state from
the restricted state temperature, gas_model.py:494-588 and 661-682), so an
RHS evaluation costs one temperature launch.  The other dependent variables
(pressure, sound speed, transport) are evaluated inside the RHS kernels and
are available here on request only.
"""

from __future__ import annotations

from dataclasses import dataclass

import torch

from mirgecom_b200 import _lib
from mirgecom_b200.eos import MixtureEOS, TemperatureSeedMissingError
from mirgecom_b200.fluid import ConservedVars


@dataclass
class GasModel:
    """mirgecom/gas_model.py:82-97."""
    eos: object
    transport: object = None

    def to_struct(self, nspecies: int) -> _lib.GasStruct:
        s = _lib.GasStruct()
        s.nspecies = nspecies
        self.eos.fill_struct(s)
        if self.transport is not None:
            self.transport.fill_struct(s, nspecies)
        else:
            s.transport_kind = _lib.TR_NONE
        return s


class FluidState:
    """mirgecom/gas_model.py:100-248 (conserved state + dependent vars).

    For the ideal gas the temperature is evaluated lazily (the RHS kernels
    compute it in registers), so building a state launches nothing.
    """

    def __init__(self, cv: ConservedVars, gas_model: GasModel, temperature=None,
                 operator_temperature=None):
        self.cv = cv
        self.gas_model = gas_model
        self._temperature = temperature
        self.operator_temperature = operator_temperature

    @property
    def temperature(self):
        if self._temperature is None:
            self._temperature = self.gas_model.eos.temperature(self.cv)
        return self._temperature

    @property
    def dim(self):
        return self.cv.dim

    @property
    def is_mixture(self):
        return isinstance(self.gas_model.eos, MixtureEOS)

    @property
    def is_viscous(self):
        return self.gas_model.transport is not None

    @property
    def mass_density(self):
        return self.cv.mass

    @property
    def momentum_density(self):
        return self.cv.momentum

    @property
    def energy_density(self):
        return self.cv.energy

    @property
    def species_mass_density(self):
        return self.cv.species_mass

    @property
    def velocity(self):
        return self.cv.velocity

    @property
    def species_mass_fractions(self):
        return self.cv.species_mass_fractions

    @property
    def pressure(self):
        eos = self.gas_model.eos
        if self.is_mixture:
            return self.cv.mass * eos.gas_const(self.cv) * self.temperature
        return eos.pressure(self.cv)

    # dependent and transport variables evaluated on the host side with torch
    # (mirgecom/gas_model.py:209-286); the operators compute their own copies
    # inside the kernels
    @property
    def speed(self):
        return self.cv.speed

    @property
    def speed_of_sound(self):
        eos = self.gas_model.eos
        if self.is_mixture:
            return eos.sound_speed(self.cv, self.temperature)
        return eos.sound_speed(self.cv)

    @property
    def wavespeed(self):
        """|v| + c (mirgecom/gas_model.py:224-226)."""
        return self.speed + self.speed_of_sound

    @property
    def viscosity(self):
        return self.gas_model.transport.viscosity(self.cv, self, self.gas_model.eos)

    @property
    def thermal_conductivity(self):
        return self.gas_model.transport.thermal_conductivity(self.cv, self, self.gas_model.eos)

    @property
    def species_diffusivity(self):
        return self.gas_model.transport.species_diffusivity(self.cv, self, self.gas_model.eos)


def make_fluid_state(cv: ConservedVars, gas_model: GasModel, temperature_seed=None,
                     **kwargs):
    """Create a thermally consistent fluid state (gas_model.py:302-430)."""
    eos = gas_model.eos
    if not isinstance(eos, MixtureEOS):
        return FluidState(cv, gas_model)
    if temperature_seed is None:
        raise TemperatureSeedMissingError("MixtureEOS.get_temperature requires a "
                                          "*temperature_seed*.")
    from mirgecom_b200 import runtime
    tseed = eos.get_temperature_seed(cv.mass, temperature_seed)
    if cv.q.dtype == torch.float32:
        # mixed form: learned guess (if the EOS carries one), float32 Newton
        # with adaptive stop, float64 residual check, plain-guess fallback
        t = runtime.mixture_temperature_mixed(cv, gas_model, tseed,
                                              iters=kwargs.get("newton_iterations"),
                                              learned=eos.learned_guess)
        return FluidState(cv, gas_model, temperature=t, operator_temperature=t)
    t1, t2 = runtime.mixture_temperature(cv, gas_model, tseed)
    return FluidState(cv, gas_model, temperature=t1, operator_temperature=t2)


def replace_fluid_state(state: FluidState, gas_model, *, mass=None, energy=None,
                        momentum=None, species_mass=None, temperature_seed=None,
                        **kwargs):
    """mirgecom/gas_model.py:907-997."""
    kw = {k: v for k, v in dict(mass=mass, energy=energy, momentum=momentum,
                                species_mass=species_mass).items() if v is not None}
    new_cv = state.cv.replace(**kw) if kw else state.cv
    tseed = temperature_seed if temperature_seed is not None else state.temperature
    return make_fluid_state(new_cv, gas_model, temperature_seed=tseed)
