// Reference header name for drop-in builds: the classes live in method.hpp.
#pragma once
#include "method.hpp"
