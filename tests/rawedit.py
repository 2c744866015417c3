"""Edits of raw event records for the error-path tests: S-Link framing faults
that the FED loop's ErrorChecker reports (ErrorChecker.cc:38-91) and extra
payload words that RawToDigi turns into error records
(SiPixelRawToClusterGPUKernel.cc:188-262).

A record is the Source's layout (Source.cc:9-21): u32 nFeds, then per FED
u32 fedId, u32 size and `size` bytes of 64-bit words (header, payload,
trailer).  Header word: low half sourceid (source id in bits 8-19, more-headers
bit 3), high half eventid (start marker 0x5 in bits 28-31).  Trailer word: low
half conscheck (CRC-modified bit 2, more-trailers bit 3), high half eventsize
(end marker 0xa in bits 28-31, length in 64-bit words in bits 0-23).
"""
import struct


def parse(raw):
    """[(fedId, [u64 words])] in record order."""
    n = struct.unpack_from("<I", raw, 0)[0]
    off, feds = 4, []
    for _ in range(n):
        fid, size = struct.unpack_from("<II", raw, off)
        off += 8
        feds.append((fid, list(struct.unpack_from("<%dQ" % (size // 8), raw, off))))
        off += size
    return feds


def build(feds):
    out = bytearray(struct.pack("<I", len(feds)))
    for fid, words in feds:
        out += struct.pack("<II", fid, 8 * len(words))
        out += struct.pack("<%dQ" % len(words), *words)
    return bytes(out)


def _fix_length(words):
    """Sets the last trailer's length field to the FED's 64-bit word count."""
    t = words[-1]
    hi = (t >> 32) & 0xffffffff
    hi = (hi & ~0x00ffffff) | (len(words) & 0x00ffffff)
    words[-1] = (hi << 32) | (t & 0xffffffff)


def crc_modified(words):
    words[-1] |= 1 << 2


def wrong_source_id(words, fed_id):
    lo = words[0] & 0xffffffff
    lo = (lo & ~0x000fff00) | ((fed_id & 0xfff) << 8)
    words[0] = (words[0] & ~0xffffffff) | lo


def extra_header(words):
    """A second header word after the first (which gets the more-headers bit)."""
    second = words[0]
    words[0] |= 1 << 3
    words.insert(1, second)
    _fix_length(words)


def bad_trailer_marker(words):
    hi = (words[-1] >> 32) & 0xffffffff
    hi = (hi & 0x0fffffff) | (0x3 << 28)
    words[-1] = (hi << 32) | (words[-1] & 0xffffffff)


def wrong_length(words, delta=3):
    hi = (words[-1] >> 32) & 0xffffffff
    hi = (hi & ~0x00ffffff) | ((len(words) + delta) & 0x00ffffff)
    words[-1] = (hi << 32) | (words[-1] & 0xffffffff)


def extra_trailer(words):
    """A second trailer word after the last.  The check starts from the FED's
    last word, so that one carries the more-trailers bit."""
    words.append(words[-1] | (1 << 3))
    _fix_length(words)
    words[-2] = (words[-2] & 0xffffffff) | (words[-1] & ~0xffffffff)


def payload32(words):
    """The 32-bit payload words between the first header and the last trailer word."""
    out = []
    for w in words[1:-1]:
        out += [w & 0xffffffff, w >> 32]
    return out


def append_payload(words, extra32):
    """Appends 32-bit payload words before the trailer (padded to an even count)."""
    extra32 = list(extra32)
    if len(extra32) % 2:
        extra32.append(0)
    pairs = [extra32[i] | (extra32[i + 1] << 32) for i in range(0, len(extra32), 2)]
    words[-1:-1] = pairs
    _fix_length(words)


def error_word(link, error_type, low=0):
    """A payload word whose ROC field carries an error type (25..31)."""
    return ((link & 0x3f) << 26) | ((error_type & 0x1f) << 21) | (low & 0x1fffff)
