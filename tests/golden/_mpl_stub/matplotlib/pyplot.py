def __getattr__(name):
    raise RuntimeError("plotting is not available in the fixture generator")
