"""Linop base-class stub: the reference's legacy Linops subclass it at import time."""


class Linop:
    def __init__(self, oshape, ishape, repr_str=None):
        self.oshape = list(oshape)
        self.ishape = list(ishape)
        self.repr_str = repr_str

    def apply(self, input):
        return self._apply(input)

    def __call__(self, input):
        return self.apply(input)


class Multiply(Linop):
    def __init__(self, ishape, mult):
        self.mult = mult
        super().__init__(ishape, ishape, "Multiply")

    def _apply(self, input):
        return input * self.mult
