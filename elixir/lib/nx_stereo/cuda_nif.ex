defmodule NxStereo.CudaNif do
  @moduledoc false
  # The NIF over libnxs_b200's C ABI (nif/nx_stereo_cuda_nif.cpp): configure
  # and run take the native Port's records (native/stereo_match/src/protocol.rs);
  # a run's reply comes as a message {ref, {:ok, outputs_record}} or
  # {ref, {:error, reason}} to the pid given.

  @on_load :load
  def load do
    path = Path.join(List.to_string(:code.priv_dir(:nx_stereo)), "nx_stereo_cuda_nif")
    case :erlang.load_nif(String.to_charlist(path), 0) do
      :ok -> :ok
      # Without the NIF (no CUDA build), CudaSegment.build/3 says so.
      {:error, _reason} -> :ok
    end
  end

  def open(_device), do: :erlang.nif_error(:not_loaded)
  def configure(_context, _record), do: :erlang.nif_error(:not_loaded)
  def run(_context, _record, _pid, _ref, _timeout_ms), do: :erlang.nif_error(:not_loaded)
  def watch(_context, _owner, _segment), do: :erlang.nif_error(:not_loaded)
  def release(_context, _segment), do: :erlang.nif_error(:not_loaded)
end
