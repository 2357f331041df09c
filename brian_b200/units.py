"""Physical units as plain SI floats.

Brian 1 scales a unit by multiplying its float value by the SI prefix factor
(fundamentalunits.py:148-150, 1123-1136), so ``1.62*mV`` is
``1.62 * 1e-3`` in double precision.  The engine runs on those same floats
(the reference's ``brian_no_units`` mode); the constants below are exactly
``1.0 * 10**k``.  Dimension checking is not performed.
"""

_PREFIXES = {"y": 1e-24, "z": 1e-21, "a": 1e-18, "f": 1e-15, "p": 1e-12, "n": 1e-9, "u": 1e-6,
             "m": 1e-3, "c": 1e-2, "d": 1e-1, "": 1.0, "da": 1e1, "h": 1e2, "k": 1e3, "M": 1e6,
             "G": 1e9, "T": 1e12, "P": 1e15, "E": 1e18, "Z": 1e21, "Y": 1e24}

_BASE = {"second": "s", "amp": "A", "volt": "V", "hertz": "Hz", "ohm": "ohm", "siemens": "S",
         "farad": "F", "metre": "m", "meter": "m", "gram": "g", "mole": "mol", "molar": "M",
         "kelvin": "K", "coulomb": "C", "newton": "N", "joule": "J", "watt": "W", "pascal": "Pa",
         "liter": "l", "litre": "l"}

__all__ = []
_g = globals()
for _name, _short in _BASE.items():
    for _p, _f in _PREFIXES.items():
        _v = float(1.0) * _f
        _long = (("deca" if _p == "da" else {"y": "yocto", "z": "zepto", "a": "atto", "f": "femto",
                  "p": "pico", "n": "nano", "u": "micro", "m": "milli", "c": "centi",
                  "d": "deci", "": "", "h": "hecto", "k": "kilo", "M": "mega", "G": "giga",
                  "T": "tera", "P": "peta", "E": "exa", "Z": "zetta", "Y": "yotta"}[_p]) + _name)
        for nm in {_p + _name, _p + _short}:
            if nm and nm not in _g and nm.isidentifier():
                _g[nm] = _v
                __all__.append(nm)
        if _long != _name and _long.isidentifier() and _long not in _g:
            _g[_long] = _v
            __all__.append(_long)
# gram is the SI-prefixed base of kilogram
kilogram = kg = 1.0
__all__ += ["kilogram", "kg"]
# units of dimensionless quantities and common aliases used in model strings
radian = 1.0
steradian = 1.0
__all__ += ["radian", "steradian"]
