from . import host, ics  # noqa: F401
