// TEST INFRASTRUCTURE ONLY: empty stand-in for an MSVC precompiled header.
#pragma once
