"""Writes the C++ blocks of the integration guide given as the first argument
(the Tracer plugin and its to_cr_config helper) to files in the directory
given as the second, so that `make -C oracle plugin-check` can compile them
against the reference's headers.  Test infrastructure."""
import os
import re
import sys

src, out = sys.argv[1], sys.argv[2]
blocks = re.findall(r"```cpp\n(.*?)```", open(src).read(), re.S)
if len(blocks) != 2:
    sys.exit(f"expected the plugin and the to_cr_config blocks, found {len(blocks)} C++ blocks")
os.makedirs(out, exist_ok=True)
for name, text in zip(("plugin.hpp", "tocfg.hpp"), blocks):
    with open(os.path.join(out, name), "w") as fh:
        fh.write(text)
