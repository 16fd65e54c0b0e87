// Forwards to the AMGCL API stand-in (shimcore.hpp).
#pragma once
#include "../shimcore.hpp"
