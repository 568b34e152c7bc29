"""ORACLE shim: import-time stand-in for pywigxjpf (used by the reference only
for the ideal bispectrum/trispectrum Fisher paths, outside this build's scope).
Test infrastructure only."""


def wig_table_init(*a, **k):
    pass


def wig_temp_init(*a, **k):
    pass


def wig3jj(*a, **k):
    raise NotImplementedError("Wigner symbols are outside the oracle's scope")


def wig6jj(*a, **k):
    raise NotImplementedError("Wigner symbols are outside the oracle's scope")
