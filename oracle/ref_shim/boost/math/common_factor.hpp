// Project-written empty stand-in: the reference includes this header but the
// filter logic compiled for the oracle uses nothing from it.
#pragma once
