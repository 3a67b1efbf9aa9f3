"""``cupy.cuda`` stand-in exposing the device attributes KSig queries."""


class _Device:
  attributes = {'MaxSharedMemoryPerBlock': 49152}

  def __init__(self, *args, **kwargs):
    pass

  def synchronize(self):
    pass


class device:  # noqa: N801 - mirrors cupy.cuda.device
  Device = _Device


Device = _Device
