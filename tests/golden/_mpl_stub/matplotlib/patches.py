class Circle:  # noqa: D101 - placeholder type for annotations
    def __init__(self, *args, **kwargs):
        pass
