#pragma once
#include "uipc_mock.h"
