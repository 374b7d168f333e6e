"""The C++ header as a host compiles it: a small program written against the reference's API names (gpu/framegen.h)
builds with include/framegen.h alone, links the library, and gets the reference's host-side answers (defaults,
validate over every Settings field with gpu/framegen.cpp:1679-1700's ranges, settingsError's refusals, formatOf,
blurPlan). Host-only calls: no GPU is needed."""
import os
import shutil
import subprocess

import pytest

REPO = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(REPO, "frame-gen-ritz_b200")

PROGRAM = r'''
#include <cstdio>
#include "framegen.h"
using namespace framegen;
#define CHECK(c) do { if (!(c)) { std::printf("FAIL %s\n", #c); return 1; } } while (0)
int main() {
    Settings d;
    CHECK(Interpolator::validate(d));
    CHECK(d.uiHistory == 3 && d.uiStillFrames == 8 && d.learnedNet == LearnedNet::E2v5 && d.v2Mode == V2Mode::Quality);
    auto bad = [](auto edit) { Settings s; edit(s); return !Interpolator::validate(s); };
    CHECK(bad([](Settings& s) { s.uiStillFrames = 0; }));
    CHECK(bad([](Settings& s) { s.uiHistory = 66; }));
    CHECK(bad([](Settings& s) { s.uiInpaintReach = 17; }));
    CHECK(bad([](Settings& s) { s.uiBoxOffsetX = -16385; }));
    CHECK(bad([](Settings& s) { s.uiCrosshairArea = 0.0f; }));
    CHECK(bad([](Settings& s) { s.v3Smear = 1.5f; }));
    CHECK(bad([](Settings& s) { s.v3OcclSoft = 0.2f; }));
    CHECK(bad([](Settings& s) { s.learnedNet = (LearnedNet)kLearnedNets; }));
    CHECK(bad([](Settings& s) { s.v3Guard = (V3Guard)3; }));
    CHECK(bad([](Settings& s) { s.trustHigh = s.trustLow + 0.5f; }));
    CHECK(!bad([](Settings& s) { s.uiReentryFrames = 0; s.uiBoxWidth = 16384; s.v3SceneCut = 4.0f; }));
    Settings v2; v2.motionVersion = MotionVersion::V2;
    CHECK(Interpolator::settingsError(v2, Format::Rgba8) != nullptr);
    Settings ui; ui.uiProtection = UiProtection::Crosshair;
    CHECK(Interpolator::settingsError(ui, Format::Rgba8) != nullptr);
    CHECK(Interpolator::settingsError(d, Format::Nv12) == nullptr);
    Format f;
    CHECK(formatOf(kVkFormatA2B10G10R10UnormPack32, &f) && f == Format::Rgb10);
    CHECK(!formatOf(12345u, &f));
    float t[16]; uint32_t q[16];
    CHECK(Interpolator::blurPlan(4, BlurWeights::Even, 0.0f, 1.0f, t, q) == 4 && q[0] == 16384 && t[0] == 0.125f);
    Interpolator fg;
    CHECK(!fg.init(InitInfo{}) && fg.initError() != nullptr);
    fg.releaseUnusedMotion();
    fg.releaseUnusedUi();
    std::printf("ok\n");
    return 0;
}
'''


@pytest.fixture(scope="module", autouse=True)
def built():
    import build
    build.build()


@pytest.mark.skipif(shutil.which("g++") is None, reason="no host C++ compiler")
def test_header_compiles_links_and_validates(tmp_path):
    src = tmp_path / "host.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "host"
    r = subprocess.run(["g++", "-std=c++17", "-O1", "-I", os.path.join(REPO, "include"), str(src), "-o", str(exe),
                        "-L", PKG, "-lframegen_b200", "-Wl,-rpath," + PKG], capture_output=True, text=True)
    assert r.returncode == 0, r.stderr[-3000:]
    r = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    assert r.returncode == 0 and r.stdout.strip() == "ok", r.stdout + r.stderr
