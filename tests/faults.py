"""A seeded event with one of each S-Link framing fault and one of each
RawToDigi error word, for the error-path tests (see rawedit.py)."""
import rawedit


def _a_link(words):
    for w in rawedit.payload32(words):
        if w and (w >> 26) & 0x3f:
            return (w >> 26) & 0x3f
    return 1


def faulted_event(det, seed, pu):
    """The event (seed, pu) with framing faults on eight FEDs and error words
    of types 25-31 (30 with both state bits) appended to two others."""
    feds = rawedit.parse(det.event(seed, pu))
    f = {i: list(w) for i, (_, w) in enumerate(feds)}
    rawedit.crc_modified(f[3])
    rawedit.wrong_source_id(f[7], feds[7][0] + 1)
    rawedit.extra_header(f[11])
    rawedit.bad_trailer_marker(f[15])
    rawedit.wrong_length(f[19])
    rawedit.extra_trailer(f[23])
    rawedit.extra_header(f[27])
    rawedit.wrong_source_id(f[27], 1201)
    rawedit.extra_trailer(f[31])
    rawedit.wrong_length(f[31], delta=-1)
    for i in (40, 41):
        link = _a_link(f[i])
        extra = [rawedit.error_word(link, 25), rawedit.error_word(link + 1, 25),
                 rawedit.error_word(link, 26, 7), rawedit.error_word(link, 27, 3), rawedit.error_word(link, 28),
                 rawedit.error_word(link, 29, (1 << 8) | 0x5), rawedit.error_word(link, 29, (4 << 8) | 0x2),
                 rawedit.error_word(link, 30, 1 << 8), rawedit.error_word(link, 30, 8 << 8),
                 rawedit.error_word(link, 30, 5 << 8), rawedit.error_word(link, 31, 0x42)]
        rawedit.append_payload(f[i], extra)
    return rawedit.build([(fid, f[i]) for i, (fid, _) in enumerate(feds)])
