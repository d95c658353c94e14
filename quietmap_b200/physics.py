"""Host-side constants of the physics, computed once in double precision.

The reference generates its device constants on the host the same way (band constants,
paint-gpu/src/device.rs:57-77); these feed scene descriptors, not the device math.
"""

import numpy as np

BAND_FREQUENCY_HZ = np.array([63.0, 125.0, 250.0, 500.0, 1000.0, 2000.0, 4000.0, 8000.0])
A_WEIGHTING_DB = np.array([-26.2, -16.1, -8.6, -3.2, 0.0, 1.2, 1.0, -1.1])
PERIOD_HOURS = np.array([12.0, 4.0, 8.0])
PERIOD_PENALTY_DB = np.array([0.0, 5.0, 10.0])


def alpha_db_per_km(frequency_hz, temperature_c, relative_humidity_pct, pressure_kpa=101.325):
    """ISO 9613-1:1993 pure-tone attenuation (dB/km), equations 3-5 with Annex B humidity
    (physics/src/atmosphere.rs:22-48)."""
    temperature = temperature_c + 273.15
    reference_temperature, triple_point = 293.15, 273.16
    pressure_ratio = pressure_kpa / 101.325
    saturation_exponent = -6.8346 * (triple_point / temperature) ** 1.261 + 4.6151
    humidity = relative_humidity_pct * 10.0 ** saturation_exponent / pressure_ratio
    oxygen = pressure_ratio * (24.0 + 4.04e4 * humidity * (0.02 + humidity) / (0.391 + humidity))
    t_ratio = temperature / reference_temperature
    nitrogen = pressure_ratio * t_ratio ** -0.5 * (
        9.0 + 280.0 * humidity * np.exp(-4.170 * (t_ratio ** (-1.0 / 3.0) - 1.0)))
    f2 = frequency_hz * frequency_hz
    return 8.686 * f2 * (
        1.84e-11 / pressure_ratio * np.sqrt(t_ratio)
        + t_ratio ** -2.5 * (0.01275 * np.exp(-2239.1 / temperature) / (oxygen + f2 / oxygen)
                             + 0.1068 * np.exp(-3352.0 / temperature) / (nitrogen + f2 / nitrogen))
    ) * 1000.0


def alpha_bands(temperature_c, relative_humidity_pct):
    """Alpha of the octave bands at exact mid-band frequencies 1000 * 10^(0.3 (k - 4))
    (physics/src/atmosphere.rs:17-19, 51-60)."""
    f = 1000.0 * 10.0 ** (0.3 * (np.arange(8) - 4.0))
    return alpha_db_per_km(f, temperature_c, relative_humidity_pct)


def lden_weights():
    """Per-period factor of the Lden energy: hours/24 * 10^(penalty/10) (bands.rs:59-66)."""
    return PERIOD_HOURS / 24.0 * 10.0 ** (PERIOD_PENALTY_DB / 10.0)
