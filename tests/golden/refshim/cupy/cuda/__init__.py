"""Stand-in for cupy.cuda: one device, streams that run in order (CPU)."""
from . import runtime  # noqa: F401


class Device:
    def __init__(self, dev=0):
        self.id = dev
        self.mem_info = (0, 1 << 40)

    def use(self):
        return None


class Stream:
    def __init__(self, *args, **kwargs):
        pass

    def use(self):
        return self

    def synchronize(self):
        return None


Stream.null = Stream()
