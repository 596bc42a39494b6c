class MaxNLocator:  # noqa: D101 - placeholder
    def __init__(self, *args, **kwargs):
        pass


class FuncFormatter:  # noqa: D101 - placeholder
    def __init__(self, *args, **kwargs):
        pass
