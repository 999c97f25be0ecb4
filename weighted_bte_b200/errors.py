"""Error contract of the weighted-BTX and weighted-PFE APIs (weighted_btx/src/error.rs:4-52;
weighted_pfe/src/error.rs:3-46 adds InvalidSecretKey and InvalidProof).

Every variant of the reference's `Error` enum is one exception class with
the same fields; all derive from `Error`.  Messages follow the reference's
`Display` strings.
"""
from __future__ import annotations


class Error(Exception):
    """Base class (the reference's `weighted_btx::Error`)."""


class BatchIsEmpty(Error):
    def __init__(self):
        super().__init__("the ciphertext batch is empty")


class BatchTooLarge(Error):
    def __init__(self, batch_size: int, max_batch_size: int):
        self.batch_size, self.max_batch_size = batch_size, max_batch_size
        super().__init__(f"batch size {batch_size} exceeds the configured maximum {max_batch_size}")


class InvalidBatchSize(Error):
    def __init__(self, size: int):
        self.size = size
        super().__init__(f"batch size {size} cannot be represented by the FFT domain")


class EmptyCommittee(Error):
    def __init__(self):
        super().__init__("the weighted committee is empty")


class InvalidPartyWeight(Error):
    def __init__(self, party_index: int, weight: int):
        self.party_index, self.weight = party_index, weight
        super().__init__(f"party {party_index} has invalid weight {weight}; every party must have positive weight")


class TotalWeightOverflow(Error):
    def __init__(self):
        super().__init__("the sum of the party weights overflows usize")


class ParameterSizeOverflow(Error):
    def __init__(self):
        super().__init__("the configured public-key dimensions overflow addressable memory")


class InvalidEvaluationDomain(Error):
    def __init__(self, total_weight: int):
        self.total_weight = total_weight
        super().__init__(f"total weight {total_weight} cannot be represented by a radix-2 scalar-field domain")


class InvalidInterpolationSet(Error):
    def __init__(self):
        super().__init__("the interpolation points must be nonempty and distinct")


class InvalidCommittee(Error):
    def __init__(self, party_count: int, total_weight: int, threshold_weight: int):
        self.party_count, self.total_weight, self.threshold_weight = party_count, total_weight, threshold_weight
        super().__init__(
            f"invalid weighted committee of {party_count} parties: threshold weight {threshold_weight} "
            f"must be smaller than total weight {total_weight}"
        )


class InvalidPartyIndex(Error):
    def __init__(self, index: int):
        self.index = index
        super().__init__(f"invalid party index {index}")


class InvalidPower(Error):
    def __init__(self, power: int, max_power: int):
        self.power, self.max_power = power, max_power
        super().__init__(f"invalid key power {power}; the supported positive magnitude is 1 through {max_power}")


class InsufficientWeight(Error):
    def __init__(self, accepted: int, required: int, rejected_parties=()):
        self.accepted, self.required = accepted, required
        self.rejected_parties = list(rejected_parties)
        msg = f"insufficient decryption weight: accepted {accepted}, require {required}"
        if self.rejected_parties:
            msg += f"; rejected parties {self.rejected_parties}"
        super().__init__(msg)


class WeightOverflow(Error):
    def __init__(self):
        super().__init__("accepted decryption weight overflows usize")


class TooManyShares(Error):
    def __init__(self, supplied: int, party_count: int):
        self.supplied, self.party_count = supplied, party_count
        super().__init__(f"too many decryption shares: supplied {supplied} for {party_count} parties")


class DuplicatePartyIndex(Error):
    def __init__(self, index: int):
        self.index = index
        super().__init__(f"duplicate party index {index}")


class MismatchedBatchSize(Error):
    def __init__(self, expected: int, actual: int):
        self.expected, self.actual = expected, actual
        super().__init__(f"mismatched batch size: expected {expected}, got {actual}")


class MismatchedBatchDigest(Error):
    def __init__(self):
        super().__init__("decryption material belongs to a different ciphertext batch")


class MismatchedSetup(Error):
    def __init__(self):
        super().__init__("cryptographic material belongs to a different setup")


class MismatchedCommittee(Error):
    def __init__(self):
        super().__init__("decryption material belongs to a different accepted committee")


class InvalidSecretKey(Error):
    def __init__(self):
        super().__init__("the party secret key produces a zero partial-fraction denominator")


class InvalidProof(Error):
    def __init__(self):
        super().__init__("the ciphertext batch contains an invalid proof")
