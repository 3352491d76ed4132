// Empty stand-in: the reference includes <boost/config.hpp> but uses nothing from it.
#pragma once
