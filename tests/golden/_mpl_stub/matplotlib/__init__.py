"""Minimal stand-in for matplotlib, used only by the fixture generator.

The reference imports matplotlib at module level for plotting; the fixture
generator never plots, so these names only need to exist.
"""


def use(*args, **kwargs):
    return None
