class Axes:  # noqa: D101 - placeholder type for annotations
    pass
