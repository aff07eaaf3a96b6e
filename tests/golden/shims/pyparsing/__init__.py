"""Import-time stand-in for ``pyparsing`` used only when generating golden fixtures.

The reference imports ``rainbow.util.parse_string`` transitively from ``rainbow.math.vector3``; that module
builds a small grammar at import time.  Nothing on the rigid-body time step parses strings, so grammar objects
here only need to survive the ``+`` / ``|`` combinators used at import.  Any attempt to actually parse raises.
"""


class _Grammar:
    def __init__(self, *args, **kwargs):
        pass

    def __add__(self, other):
        return self

    __radd__ = __add__
    __or__ = __add__
    __ror__ = __add__

    def parse_string(self, *args, **kwargs):
        raise RuntimeError("string parsing is not available in the golden-fixture environment")

    parseString = parse_string


Regex = Word = LineEnd = Literal = Optional = Suppress = Combine = _Grammar


def delimitedList(*args, **kwargs):
    return _Grammar()


delimited_list = delimitedList
alphas = "abcdefghijklmnopqrstuvwxyzABCDEFGHIJKLMNOPQRSTUVWXYZ"
nums = "0123456789"
