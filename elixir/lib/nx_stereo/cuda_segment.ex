defmodule NxStereo.CudaSegment do
  @moduledoc """
  A list of stages computed on an NVIDIA B200 by nx_stereo_b200's CUDA
  kernels, run on each pair as one request: a drop-in for
  `NxStereo.NativeSegment` with the same stages, settings, params, entries
  and outputs (lib/nx_stereo/native_segment.ex:1-43), through the NIF
  `NxStereo.CudaNif` instead of the `stereo_match` Port.

  The NIF takes the very records NativeSegment sends its Port: a segment's
  configuration (each stage's kind, build settings and native constants),
  and per pair each stage's params and the entries. Requests on a segment
  are computed in the order sent; a segment whose stages carry nothing
  from pair to pair computes neighbouring pairs at once on two device
  streams, and one that does (TemporalFilter, Quality) one after another.
  Up to `depth/0` pairs may be at the device at once.

  Building does not reach the device: the segment is configured on its
  first pair and again after `reload/3`. A configuration the library
  refuses answers that pair with `{:stop, reason}`. A run without a reply
  within `:timeout_ms` (build option, 5000) fails with `{:error, :timeout}`,
  and so does every run sent after it, as `NxStereo.Matcher` fails the
  requests waiting behind a late reply. The process that builds the
  segment owns it: the device releases it once that process exits.
  """

  @behaviour NxStereo.Segment

  alias NxStereo.{CudaNif, Segment, Stage}

  @enforce_keys [:context, :id, :version, :members, :specs, :geometry]
  defstruct [
    :context,
    :owner,
    :id,
    :version,
    :configured_version,
    :members,
    :specs,
    :geometry,
    :configuration,
    :inputs,
    timeout_ms: 5_000,
    times_us: []
  ]

  @configure 1
  @run 2
  @type_codes %{{:u, 8} => 0, {:u, 16} => 1, {:f, 32} => 2, {:s, 32} => 3}
  @types Map.new(@type_codes, fn {type, code} -> {code, type} end)

  @impl Segment
  def compute(%__MODULE__{}), do: %{runs_on: :gpu, implementation: :cuda, backend: nil}

  @doc "Four pairs: copies, kernels and replies of neighbouring pairs overlap on the device."
  @impl Segment
  def depth, do: 4

  @doc "As NativeSegment: a native kind, and settings that do not ask for Nx."
  @impl Segment
  def accepts?(module, state, compute),
    do: compute == :native and refusal(%{module: module, state: state}) == nil

  @doc """
  The segment of `members` for `geometry`, with `opts`: `:device` (0), the
  CUDA device, and `:timeout_ms` (5000), how long a pair may wait for its
  reply.
  """
  @impl Segment
  def build(members, geometry, opts) do
    with {:ok, opts} <- validate(opts),
         nil <- Enum.find_value(members, &refusal/1),
         {:ok, specs} <- Segment.entry_specs(members, geometry),
         {:ok, context} <- context(opts[:device]) do
      segment = %__MODULE__{
        context: context,
        owner: self(),
        id: rem(System.unique_integer([:positive]), 0x1_0000_0000),
        version: 0,
        members: members,
        specs: specs,
        geometry: geometry,
        timeout_ms: opts[:timeout_ms]
      }

      {:ok, prepare(segment)}
    end
  end

  defp validate(opts) do
    case Keyword.validate(opts, device: 0, timeout_ms: 5_000) do
      {:ok, opts} -> {:ok, opts}
      {:error, unknown} -> {:error, "unknown build options #{inspect(unknown)}"}
    end
  end

  # One context a device for the whole node, opened on first use.
  defp context(device) do
    key = {__MODULE__, device}

    case :persistent_term.get(key, nil) do
      nil ->
        case CudaNif.open(device) do
          {:ok, context} ->
            :persistent_term.put(key, context)
            {:ok, context}

          {:error, reason} ->
            {:error, "no CUDA device #{device}: #{reason}"}
        end

      context ->
        {:ok, context}
    end
  rescue
    ErlangError -> {:error, "the nx_stereo_b200 NIF is not loaded"}
  end

  defp refusal(%{module: module, state: state}) do
    cond do
      Stage.native_kind(module) == nil ->
        {:error, "#{inspect(module)} has no native implementation"}

      Stage.compute(module, state) == :nx ->
        {:error, "#{inspect(module)} is computed in Nx, as its settings ask"}

      true ->
        nil
    end
  end

  @impl Segment
  def reload(%__MODULE__{} = segment, members, geometry),
    do: prepare(%{segment | members: members, geometry: geometry, version: segment.version + 1})

  @impl Segment
  def put_member_state(%__MODULE__{members: members} = segment, index, state) do
    members = List.update_at(members, index, &%{&1 | state: state})
    %{segment | members: members, inputs: inputs(members, segment.geometry)}
  end

  @doc "`current`: the device keeps what the stages carry."
  @impl Segment
  def merge_carry(%__MODULE__{} = current, %__MODULE__{}), do: current

  @doc """
  Hands a pair's `entries` to the device without waiting; returns the
  reference its reply comes back with. The segment is configured first
  when its version changed (a first pair, a reload).
  """
  @impl Segment
  def send_request(entries, %__MODULE__{} = segment) do
    with {:ok, entry} <- Segment.entry_tensors(entries, segment.specs),
         :ok <- configure(segment) do
      ref = make_ref()
      record = IO.iodata_to_binary([<<@run, segment.id::little-32>>, segment.inputs, encode(entry)])

      case CudaNif.run(segment.context, record, self(), ref, segment.timeout_ms) do
        :ok -> {:ok, ref}
        {:error, reason} -> {:ok, {:failed, ref, reason}}
      end
    else
      {:refused, reason} -> {:ok, {:refused, reason}}
      error -> error
    end
  end

  # The version the device has is kept in the process that owns the segment.
  defp configure(%__MODULE__{id: id, version: version} = segment) do
    key = {__MODULE__, :configured, id}

    if Process.get(key) == version do
      :ok
    else
      case CudaNif.configure(segment.context, segment.configuration) do
        :ok ->
          CudaNif.watch(segment.context, segment.owner, id)
          Process.put(key, version)
          :ok

        {:error, {:configuration_refused, reason}} ->
          {:refused, reason}

        {:error, reason} ->
          {:refused, reason}
      end
    end
  end

  @impl Segment
  def response(message, request, %__MODULE__{} = segment) do
    case {message, request} do
      {_, {:refused, reason}} -> {:stop, reason}
      {_, {:failed, _ref, reason}} -> {:error, reason}
      {{ref, reply}, ref} -> received(reply, segment)
      _ -> :no_reply
    end
  end

  @impl Segment
  def await({:refused, reason}, _segment, _timeout), do: {:stop, reason}
  def await({:failed, _ref, reason}, _segment, _timeout), do: {:error, reason}

  def await(ref, %__MODULE__{} = segment, timeout) do
    receive do
      {^ref, reply} -> received(reply, segment)
    after
      timeout -> :timeout
    end
  end

  defp received({:ok, <<8, rest::binary>>}, segment) do
    case decode(rest) do
      {:ok, times_us, outputs} ->
        {:ok, outputs, %{segment | times_us: times_us}, System.monotonic_time(:nanosecond)}

      error ->
        error
    end
  end

  defp received({:error, reason}, _segment), do: {:error, reason}

  @impl Segment
  def member_times(%__MODULE__{members: members, times_us: times_us}),
    do: Enum.zip_with(members, times_us, &{&1.name, &2 * 1_000})

  @impl Segment
  def collect(outputs, %__MODULE__{}, _timeout), do: {:ok, outputs}

  # -- the records, as the native Port takes them (protocol.rs:1-23)

  defp prepare(segment),
    do: %{
      segment
      | configuration: configuration(segment),
        inputs: inputs(segment.members, segment.geometry)
    }

  defp configuration(%__MODULE__{id: id, members: members, geometry: g}) do
    IO.iodata_to_binary([
      <<@configure, id::little-32, g.width::little-16, g.height::little-16,
        g.frame_width::little-16, g.frame_height::little-16, length(members)>>,
      for %{module: module, state: state} <- members do
        settings =
          Stage.native_settings(module, state) ++ Enum.sort(Stage.native_constants(module))

        [
          name(module.native_kind()),
          length(settings),
          for({key, value} <- settings, do: [name(key), <<number(value)::little-float-64>>])
        ]
      end
    ])
  end

  defp number(true), do: 1.0
  defp number(false), do: 0.0
  defp number(value), do: value * 1.0

  defp inputs(members, geometry) do
    IO.iodata_to_binary([
      length(members),
      for %{module: module, state: state} <- members do
        values = module |> Stage.params(state, geometry) |> flatten("") |> Enum.sort()

        [
          length(values),
          for({key, f32} <- values, do: [name(key), <<div(byte_size(f32), 4)::little-16>>, f32])
        ]
      end
    ])
  end

  defp flatten(params, prefix) do
    Enum.flat_map(params, fn
      {key, %Nx.Tensor{} = t} -> [{prefix <> to_string(key), t |> Nx.as_type(:f32) |> Nx.to_binary()}]
      {key, v} when is_number(v) -> [{prefix <> to_string(key), <<v::little-float-32>>}]
      {key, %{} = nested} -> flatten(nested, "#{prefix}#{key}.")
    end)
  end

  defp name(key) do
    key = to_string(key)
    [byte_size(key), key]
  end

  defp encode(entry) do
    [
      length(entry),
      for {field, tensor} <- entry do
        {height, width} = Nx.shape(tensor)

        [
          name(field),
          <<Map.fetch!(@type_codes, Nx.type(tensor)), 2, height::little-32, width::little-32>>,
          Nx.to_binary(tensor)
        ]
      end
    ]
  end

  defp decode(<<count, times::binary-size(count * 4), n, rest::binary>>) do
    times_us = for <<t::little-32 <- times>>, do: t
    with {:ok, outputs} <- tensors(n, rest, %{}), do: {:ok, times_us, outputs}
  end

  defp decode(_), do: {:error, :bad_reply}

  defp tensors(0, <<>>, outputs), do: {:ok, outputs}

  defp tensors(n, <<length, key::binary-size(length), code, rank, rest::binary>>, outputs)
       when is_map_key(@types, code) do
    <<dims::binary-size(rank * 4), rest::binary>> = rest
    shape = for <<d::little-32 <- dims>>, do: d
    {_, bits} = type = Map.fetch!(@types, code)
    size = Enum.product(shape) * div(bits, 8)
    <<data::binary-size(size), rest::binary>> = rest
    tensor = data |> Nx.from_binary(type, backend: Nx.BinaryBackend) |> Nx.reshape(List.to_tuple(shape))
    tensors(n - 1, rest, Map.put(outputs, String.to_existing_atom(key), tensor))
  end

  defp tensors(_, _, _), do: {:error, :bad_reply}
end
