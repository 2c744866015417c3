"""The chain's modules inside the reference's own event processor
(src/serial/bin/EventProcessor.cc and Framework/, built from its sources by
oracle/ref/Makefile target fw; driver oracle/ref/fw_main.cc):
SiPixelRawToClusterCUDA, SiPixelRecHitCUDA, CAHitNtupletCUDA and
PixelVertexProducerCUDA with the transfer modules (SiPixelDigisSoAFromCUDA,
PixelTrackSoAFromCUDA, PixelVertexSoAFromCUDA) and the four ESProducers,
loaded by name from plugins.txt out of pluginPixelB200.so, and the
reference's serial CountValidator (plugin-Validation/CountValidator.cc)
checking the products against the oracle's counts (digicluster.bin,
tracks.bin, vertices.bin): modules, digis and clusters exactly, tracks
within 1.2 %, vertices within 1.  Several concurrent events share the
chain's batches."""
import os
import re
import subprocess

import pytest

pytestmark = pytest.mark.gpu
ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
EXE = os.path.join(ROOT, "oracle", "_ref", "fw", "edm_b200")


@pytest.fixture(scope="module")
def data_dir(tmp_path_factory, default_detector):
    import pixgpu
    import fwdata
    d = str(tmp_path_factory.mktemp("fwdata"))
    raws = [default_detector.event(pixgpu.BENCH_SEED_BASE + k, 50, model=pixgpu.BENCH_MODEL) for k in range(24)]
    raws += [default_detector.event(pixgpu.BASE_SEED + 50 + k, 20) for k in range(8)]
    want = fwdata.write_data_dir(d, default_detector, raws)
    return d, want


@pytest.mark.skipif(not os.path.exists(EXE), reason="the framework checker build needs the reference tree")
@pytest.mark.parametrize("streams", [1, 4])
def test_event_processor_with_b200_plugins_validates(data_dir, streams):
    d, want = data_dir
    r = subprocess.run([EXE, "--data", d, "--validation", "--numberOfStreams", str(streams)], capture_output=True,
                       text=True, timeout=600)
    assert r.returncode == 0, r.stdout[-3000:] + r.stderr[-3000:]
    assert "CountValidator: all %d events passed validation" % len(want) in r.stdout, r.stdout[-3000:]
    # exact counts: the validator reports any track or vertex difference it tolerated
    assert "Average relative track difference" not in r.stdout
    assert "Average absolute vertex difference" not in r.stdout
    assert re.search(r"Processed %d events" % len(want), r.stdout)
