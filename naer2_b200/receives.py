"""Annotation markers of hook parameters (reference naer2/receives.py): a hook
declares which of the framework's values it takes by annotating a parameter
with one of these types."""


class time:
    """The hook's time (ms): the end of the step it runs in."""


class edge:
    """The link being delivered (receive): edge.<attr> reads a per-link attribute."""


class source:
    """The sending neuron of the link being delivered."""


class destination:
    """The receiving neuron of the link being delivered (edge hooks)."""


__all__ = ["time", "edge", "source", "destination"]
