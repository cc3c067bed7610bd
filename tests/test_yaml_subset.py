"""The YAML-subset header that stands in for yaml-cpp when the reference's
driver is built on this library (oracle/yaml_subset): block maps and
sequences, flow sequences and maps, comments, quoted scalars, missing keys,
conversions and their errors, as a C++ program compiled against it sees them."""
import os
import shutil
import subprocess

import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROGRAM = r'''
#include <iostream>
#include <set>
#include <yaml-cpp/yaml.h>
int main(int argc, char** argv) {
    const YAML::Node r = YAML::LoadFile(argv[1]);
    const YAML::Node g = r["general"];
    std::cout << g["Element"].as<std::string>() << " " << g["a0"].as<double>() << " " << g["Nx"].as<int>()
              << " " << (bool)g["Missing"] << " " << r["dislocations"].size() << " "
              << r["dislocations"].IsSequence() << " " << g.IsMap() << "\n";
    const YAML::Node d = r["dislocations"][1];
    std::cout << d["Shape"].as<std::string>() << " " << d["Center"].size() << " " << d["Center"][2].as<double>()
              << " " << d["m"][0].as<int>() << "\n";
    std::set<std::string> keys;
    for (const auto& kv : g) keys.insert(kv.first.as<std::string>());
    std::cout << keys.size() << "\n";
    const YAML::Node f = YAML::Load("a: {X: [1, -1, 0], Y: [[1, 2], [3, 4]]}  # c\nb: 'q # not a comment'\n"
                                    "c:\n- 1\n- two\n-\n  - 3\nd: ~\n");
    std::cout << f["a"]["X"][1].as<int>() << " " << f["a"]["Y"][1][0].as<int>() << " "
              << f["b"].as<std::string>() << "|" << f["c"].size() << " " << f["c"][1].as<std::string>() << " "
              << f["c"][2][0].as<int>() << " " << f["d"].IsNull() << "\n";
    try { f["c"][1].as<double>(); std::cout << "no error\n"; }
    catch (const YAML::Exception&) { std::cout << "bad conversion\n"; }
    const YAML::Node empty = r["nope"] ? r["nope"] : YAML::Node(YAML::NodeType::Sequence);
    std::cout << empty.IsSequence() << " " << empty.size() << "\n";
    try { YAML::LoadFile("/nonexistent.yaml"); } catch (const YAML::Exception&) { std::cout << "bad file\n"; }
    return 0;
}
'''


def test_yaml_subset(tmp_path):
    cxx = os.environ.get("DISCO_CXX", "g++")
    if shutil.which(cxx) is None:
        pytest.skip("no C++ compiler")
    src = tmp_path / "y.cpp"
    src.write_text(PROGRAM)
    exe = tmp_path / "y"
    subprocess.run([cxx, "-std=c++14", "-I", os.path.join(ROOT, "oracle", "yaml_subset"), str(src), "-o", str(exe)],
                   check=True)
    out = subprocess.run([str(exe), os.path.join(ROOT, "tests", "data", "quadrupole_small.yaml")],
                         capture_output=True, text=True, check=True).stdout.splitlines()
    assert out == ["Fe 2.855 20 0 4 1 1", "circular 3 0 -1", "9",
                   "-1 3 q # not a comment|3 two 3 1", "bad conversion", "1 0", "bad file"]
