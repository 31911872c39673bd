// Per-net constants handed to every model function (spice/snn_info.h:8-14).
#pragma once

namespace spice
{
struct snn_info
{
	int num_neurons = 0;
};
} // namespace spice
