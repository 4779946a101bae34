#pragma once
#include "gadgetron_stub.h"
