"""Luminosity distance in the Planck 2018 cosmology, for pe_redshift's z grid.

The reference takes D_L(z) from astropy.cosmology.Planck18 (exmarg/search/pe.py:26-28), which is not
installed here.  This module restates that cosmology from its published parameters (Planck 2018,
TT,TE,EE+lowE+lensing+BAO, as astropy tabulates them: H0 = 67.66 km/s/Mpc, Om0 = 0.30966 in
non-relativistic matter other than neutrinos, Tcmb0 = 2.7255 K, Neff = 3.046, neutrino masses
0, 0, 0.06 eV, spatially flat) and the same treatment of the radiation:

* photons: Omega_gamma0 = 4 sigma_SB Tcmb0^4 / (c^3 rho_crit0), rho_crit0 = 3 H0^2 / (8 pi G);
* neutrinos: their density relative to the photons' is 7/8 (4/11)^(4/3) Neff/3 times, per
  species, 1 for a massless one and (1 + (k y)^p)^(1/p) for a massive one (k = 0.3173,
  p = 1.83, y = m / (k_B T_nu0 (1 + z)), T_nu0 = (4/11)^(1/3) Tcmb0; Komatsu et al. 2011,
  ApJS 192, 18, eq. 26);
* dark energy: a cosmological constant closing the budget.

D_L(z) = (1 + z) (c / H0) int_0^z dz' / E(z'),  E^2 = Om0 (1+z)^3 + Og0 (1+z)^4 (1 + nu(z)) + OL.
Physical constants are CODATA 2018 and the IAU 2015 parsec.
"""

import numpy as np
from scipy import integrate

C_KMS = 299792.458                 # km/s
C_MS = 299792458.0                 # m/s
G_SI = 6.67430e-11                 # m^3 kg^-1 s^-2
SIGMA_SB = 5.670374419e-8          # W m^-2 K^-4
K_B_EV = 8.617333262e-5            # eV / K
MPC_M = 3.0856775814913673e22      # m

PLANCK18 = dict(H0=67.66, Om0=0.30966, Tcmb0=2.7255, Neff=3.046, m_nu=(0.0, 0.0, 0.06))


class FlatLCDMNu:
    """flat Lambda-CDM with photons and three neutrino species (massless or massive)"""

    def __init__(self, H0, Om0, Tcmb0, Neff, m_nu):
        self.H0, self.Om0, self.Tcmb0, self.Neff = float(H0), float(Om0), float(Tcmb0), float(Neff)
        m_nu = np.asarray(m_nu, float)
        h0_si = self.H0 * 1e3 / MPC_M                               # 1/s
        rho_crit = 3.0 * h0_si ** 2 / (8.0 * np.pi * G_SI)           # kg / m^3
        self.Og0 = 4.0 * SIGMA_SB * self.Tcmb0 ** 4 / C_MS ** 3 / rho_crit
        t_nu0 = (4.0 / 11.0) ** (1.0 / 3.0) * self.Tcmb0
        self._massive = m_nu > 0
        self._nu_y = m_nu[self._massive] / (K_B_EV * t_nu0)
        self._n_massless = int(np.sum(~self._massive))
        self._nu_prefac = 7.0 / 8.0 * (4.0 / 11.0) ** (4.0 / 3.0) * self.Neff / m_nu.size
        self.Onu0 = self.Og0 * self.nu_relative_density(0.0)
        self.Ode0 = 1.0 - self.Om0 - self.Og0 - self.Onu0
        self.hubble_distance = C_KMS / self.H0                      # Mpc

    def nu_relative_density(self, z):
        """neutrino energy density over the photons' at redshift z"""
        z = np.asarray(z, float)
        k, p = 0.3173, 1.83
        y = self._nu_y[:, None] / (1.0 + np.atleast_1d(z))[None, :] if self._nu_y.size else np.zeros((0, 1))
        rel = np.sum((1.0 + (k * y) ** p) ** (1.0 / p), axis=0) + self._n_massless
        out = self._nu_prefac * rel
        return out if z.ndim else float(out[0])

    def efunc(self, z):
        z = np.asarray(z, float)
        zp1 = 1.0 + z
        return np.sqrt(self.Om0 * zp1 ** 3 + self.Og0 * zp1 ** 4 * (1.0 + self.nu_relative_density(z)) + self.Ode0)

    def comoving_distance(self, z):
        """Mpc, adaptive quadrature of 1/E per redshift (relative accuracy ~1e-12)"""
        z = np.atleast_1d(np.asarray(z, float))
        f = lambda x: 1.0 / float(self.efunc(x))
        out = np.array([integrate.quad(f, 0.0, zi, epsabs=0.0, epsrel=1e-12, limit=200)[0] if zi > 0 else 0.0
                        for zi in z])
        return self.hubble_distance * out

    def luminosity_distance(self, z):
        """Mpc"""
        z = np.atleast_1d(np.asarray(z, float))
        return (1.0 + z) * self.comoving_distance(z)


planck18 = FlatLCDMNu(**PLANCK18)


def dl_of_z(z):
    """luminosity distance (Mpc) at each redshift, Planck 2018 (exmarg/search/pe.py:26-28)"""
    return planck18.luminosity_distance(z)
