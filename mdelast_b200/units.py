"""CGS unit constants of mdelast (``src/units.hpp:6-24``), the units of every quantity
that crosses the ``md_driver_module`` boundary."""


class Units:
    k_boltz = 1.38064852e-16
    Navogadro = 6.02214086e23  # mol-1
    ev = 1.6021773e-12
    joule = 1e7
    angstrom = 1e-8
    nm = 1e-7
    bar = 1e6
    kbar = 1e3 * bar
    atm = 1.01325 * bar
    Pa = 1e-5 * bar
    GPa = 1e9 * Pa
    mus = 1e-6
    ns = 1e-9
    ps = 1e-12
    fs = 1e-15
