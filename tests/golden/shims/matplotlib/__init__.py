"""No-op matplotlib stand-in: the reference imports it for plots only."""


def use(*args, **kwargs):
    return None
